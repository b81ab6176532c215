// Wavefront path tracer kernels.
//
// The reference runs one thread per pixel with a 64-byte PathState reloaded each bounce
// (Render / RenderIteration, src/Shaders/kernels/testrenderer.slang:1087-1144) and appends
// deferred shadow rays for one ProcessShadowRays pass (:296-323, :1147-1166).  Here every bounce
// is three kernels over compacted structure-of-arrays queues:
//   extend  -- closest-hit BVH8 traversal of the live path queue (persistent, warp work fetch)
//   shade   -- hit reconstruction, emission + MIS, NEE light sample, Russian roulette and BSDF
//              sampling; survivors are appended to the next queue and shadow rays to the shadow
//              queue with warp-aggregated atomics
//   occlude -- first-hit traversal of the shadow queue, adding unoccluded contributions
// A wave holds `pixels x slots` camera paths; path p owns accumulator slot p, so every
// accumulator element has exactly one writer per kernel and needs no atomics: the summation
// order is fixed and results are deterministic.
#pragma once
#include "s2_hashgrid.cuh"
#include "s2_lights.cuh"
#include "s2_traverse.cuh"

namespace s2 {

enum Counter : uint32_t {
    C_QUEUE0 = 0,   // live paths in queue 0 / 1 (by bounce parity)
    C_QUEUE1 = 1,
    C_SHADOW = 2,   // shadow rays appended this bounce
    C_WORK_EXT = 3, // warp work counters for the persistent traversal kernels
    C_WORK_OCC = 4,
    C_CACHEQ = 5,   // radiance-cache queries appended this bounce
    C_TRAIN = 6,    // radiance-cache training vertices appended this wave
    C_SHADOW1 = 7,  // shadow rays of odd bounces when shadow tracing is merged into the next trace
    C_COUNT = 8
};
enum Stat : uint32_t { S_EXT = 0, S_SHADOW = 1, S_NAN = 2, S_EXT_NODES = 3, S_EXT_TRIS = 4, S_SH_NODES = 5, S_SH_TRIS = 6, S_COUNT = 8 };

struct PathQueue { float4* s0; float4* s1; float4* s2; uint4* s3; };

// One view of a batched (multi-view) render: ViewData + camera transform, its slice of the path
// space (path_offset .. path_offset + pixels * spp), its slice of the concatenated per-pixel
// accumulators (pixel_offset), and its AOV outputs.
struct ViewEntry {
    float proj[8];
    int imin[2], imax[2];
    float cam[12];
    float prev_inv[12];
    uint32_t width, height, pixels, pixel_offset;
    unsigned long long path_offset;
    float4* aov_albedo;
    uint2* aov_vis;
    float4* aov_depth;
    float2* aov_prev_uv;
    uint2* aov_ids;
};

struct PTParams {
    DevScene scene;
    // view (ViewData + camera transform)
    float proj[8];
    int imin[2], imax[2];
    float cam[12];
    float prev_inv[12];
    uint32_t width, height, pixels;
    // render parameters
    uint32_t min_len, max_len, flags, frame_seed, restir_m;
    float exposure;
    // wave
    uint32_t wave_base_sample, wave_samples;
    // buffers
    PathQueue q[2];
    float4* hits;
    float4 *sh_o, *sh_d, *sh_c;
    float4* accum;
    uint32_t* counters;
    unsigned long long* stats;
    int* status;
    // AOVs (device, may be null)
    float4* aov_albedo;
    uint2* aov_vis;
    float4* aov_depth;
    float2* aov_prev_uv;
    uint2* aov_ids;
    // batched streaming mode (s2_render_views): view table, fixed-point per-pixel accumulators,
    // path-space size and queue capacity; null / 0 in wave mode
    const ViewEntry* views;
    uint32_t nviews, view_spp;
    unsigned long long image_paths;  // batched: paths of the views; ids beyond are training paths
    uint32_t batch_pixels;
    unsigned long long* total_fx;   // 4 x u64 per pixel: r, g, b fixed point (2^-24), unused
    unsigned long long total_paths;
    uint32_t capacity;
    unsigned long long* stream_state; // [0] next path id, [1] regen base, [2] regen count, [3] done
    // ReSTIR DI reuse through the world-space hash grids (S2_FLAG_RESTIR_REUSE)
    HashGridDev grid_cur, grid_prev;
    uint32_t reuse, prev_valid;
    float max_m;
    // screen-space ReSTIR DI reuse (S2_FLAG_RESTIR_SCREEN): per-pixel reservoirs of the previous
    // call (read) and of this call (written by each pixel's sample-0 primary vertex)
    const ReservoirRecord* ss_prev;
    ReservoirRecord* ss_cur;
    uint32_t ss_on, ss_prev_valid, ss_spatial;
    float ss_radius;
    // learned radiance cache (S2_FLAG_RADIANCE_CACHE): non-training paths end at vertex cache_len
    // with a query {position, slot} + throughput; training paths (meta bit 9, one in train_mod)
    // record every vertex {position, slot}, throughput, accumulated radiance
    uint32_t cache_on, cache_len, train_mod;
    // path regularisation of the cache form: the roughness of every vertex after the first is raised
    // to at least cache_rough; 0 = off
    float cache_rough;
    float4 *cq_pos, *cq_thr;
    uint32_t cq_cap;
    float4 *tr_pos, *tr_thr, *tr_rad;
    uint32_t tr_cap;
    // traversal tuning (s2_autotune / s2_set_tuning; 0 = default)
    TravTuning trav;
    uint32_t refill_min;  // refill a warp's idle lanes once this many are idle
    // material-key sorting before shading (S2Tuning::shade_order): k_extend writes a key per
    // path (hit material, misses last), a counting sort builds sort_perm, k_shade reads through it
    // light tracing (S2_FLAG_LIGHT_TRACE): world-to-camera transform, light subpaths per pass and
    // the image-plane distance of ViewData::imagePlaneDist
    float cam_inv[12];
    uint32_t lt_paths;
    float lt_image_plane_dist;
    uint32_t sort_on;
    // ray-coherence sorting before traversal (S2Tuning::trace_order): k_shade writes ray_key() of
    // each continuation ray (ray_sort_on), a counting sort builds sort_perm, and k_extend takes its
    // rays through it (ray_sorted, set per launch)
    uint32_t ray_sort_on, ray_sorted;
    uint32_t* sort_keys;
    uint32_t* sort_perm;
    uint32_t* sort_hist;   // kSortBuckets counters / offsets
    // camera launches of frames with several samples per pixel: the triangle hit by each pixel's
    // centre ray (k_pixel_hint), tested first so that the traversal starts with a tight t_max
    const uint32_t* hint_tri;
    // shadow rays traced by the next bounce's k_trace (S2Tuning::shadow_merge): the shade kernel
    // counts its shadow rays in C_SHADOW1 when sh_parity is 1, so that the previous bounce's count
    // stays readable while they are traced; sh_merge tells k_bounce_setup which count to retire
    uint32_t sh_parity, sh_merge;
};

__host__ __device__ __forceinline__ uint32_t sh_counter(const PTParams& P) { return P.sh_parity ? C_SHADOW1 : C_SHADOW; }

constexpr uint32_t kSortBuckets = 4096;  // k_sort_scan: 1024 threads x 4 buckets


// Adds a contribution to a path's accumulator: an exclusive float slot in wave mode, or an atomic
// fixed-point add into the pixel's total in batched mode.
// Batched mode: pixel slots accumulate in fixed point; slots with bit 31 set are radiance-cache
// training paths, which accumulate their own radiance in accum[slot & 0x7fffffff] (the training
// targets need it per path) and add nothing to the image.
constexpr uint32_t kTrainSlot = 0x80000000u;
S2D void add_contrib(const PTParams& P, uint32_t slot, float3 v) {
    if (P.total_fx && (slot & kTrainSlot)) {
        float* a = (float*)(P.accum + (slot & ~kTrainSlot));
        atomicAdd(a + 0, v.x); atomicAdd(a + 1, v.y); atomicAdd(a + 2, v.z);
        return;
    }
    if (P.total_fx) {
        unsigned long long* t = P.total_fx + 4 * (size_t)slot;
        if (v.x > 0.f) atomicAdd(t + 0, (unsigned long long)__float2ull_rn(v.x * S2_FX_SCALE));
        if (v.y > 0.f) atomicAdd(t + 1, (unsigned long long)__float2ull_rn(v.y * S2_FX_SCALE));
        if (v.z > 0.f) atomicAdd(t + 2, (unsigned long long)__float2ull_rn(v.z * S2_FX_SCALE));
        return;
    }
    float4 a = P.accum[slot];
    a.x += v.x; a.y += v.y; a.z += v.z;
    P.accum[slot] = a;
}

#define S2F_JITTER (1u << 0)
#define S2F_LAMBERT (1u << 1)
#define S2F_PCG32 (1u << 2)
#define S2F_NO_NEE (1u << 3)
#define S2F_RESTIR (1u << 4)
#define S2F_REF_ENV_MIS (1u << 5)
#define S2F_NO_RR (1u << 6)
#define S2F_NO_SN (1u << 8)
#define S2F_REUSE (1u << 11)
#define S2F_SCREEN (1u << 15)
#define S2F_NO_ALPHA (1u << 12)
#define S2F_NO_NORMAL_MAPS (1u << 13)
#define S2F_CACHE (1u << 14)
#define S2F_REUSE_VIS (1u << 18)

constexpr int kTravBlock = 128;


// ---------------------------------------------------------------- camera rays
// InitializeCameraPath (testrenderer.slang:938-957): ViewData::toWorld (compat/scene.h:152-157)
// through ProjectionData::backProject (compat/transform.h:159-170); the direction is stored
// octahedral-packed as the reference's PathState.mRayDirection is.
// Camera ray through pixel (px, py) (+ offset) of a view: InitializeCameraPath
// (testrenderer.slang:938-957), ViewData::toWorld / ProjectionData::backProject.
S2D float3 camera_dir(const float* proj, const int* imin, const int* imax, const float* c, uint32_t px, uint32_t py,
                      float ox, float oy) {
    const float W = (float)(imax[0] - imin[0]), H = (float)(imax[1] - imin[1]);
    const float uvx = ((float)px + ox - imin[0]) / W, uvy = ((float)py + oy - imin[1]) / H;
    const float cx = 2.f * uvx - 1.f, cy = -(2.f * uvy - 1.f);
    const float sx = proj[0], sy = proj[1], offx = proj[2], offy = proj[3], nr = proj[4];
    float3 ld;
    if (proj[7] < 0.f) ld = f3((cx - offx) / sx, (cy - offy) / sy, nr);
    else {
        const float sg = nr > 0.f ? 1.f : (nr < 0.f ? -1.f : 0.f);
        ld = f3(nr * (cx * sg - offx) / sx, nr * (cy * sg - offy) / sy, nr);
    }
    ld = normalize(ld);
    const float3 wd = normalize(f3(c[0] * ld.x + c[1] * ld.y + c[2] * ld.z, c[4] * ld.x + c[5] * ld.y + c[6] * ld.z,
                                   c[8] * ld.x + c[9] * ld.y + c[10] * ld.z));
    return unpack_normal(pack_normal(wd));
}

__global__ void k_raygen(PTParams P) {
    const uint32_t n = P.pixels * P.wave_samples;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        P.counters[C_QUEUE0] = n;
        P.counters[C_QUEUE1] = 0;
        P.counters[C_SHADOW] = 0;
        P.counters[C_SHADOW1] = 0;
        P.counters[C_WORK_EXT] = 0;
        P.counters[C_WORK_OCC] = 0;
        P.counters[C_CACHEQ] = 0;
        P.counters[C_TRAIN] = 0;
    }
    if (i >= n) return;
    // Queue order: pixel (row-major), then sample.  A warp takes 32 samples of one pixel (or, with
    // fewer samples per wave, the samples of neighbouring pixels): camera rays through one pixel
    // visit nearly the same BVH nodes, so the warp's lanes step through the traversal together,
    // and the pixels in flight at any time cover a few image rows, whose BVH region stays in L2.
    // The accumulator slot keeps the sample-major layout that k_reduce sums.
    const uint32_t pix = i / P.wave_samples, k = i - pix * P.wave_samples;
    const uint32_t py = pix / P.width, px = pix - py * P.width;
    const uint32_t slot = k * P.pixels + pix;
    const uint32_t sample = P.wave_base_sample + k;
    Rng rng = make_rng(px, py, P.frame_seed + sample, (P.flags & S2F_PCG32) != 0);
    float ox = 0.5f, oy = 0.5f;
    if (P.flags & S2F_JITTER) { const float4 f = rng.next_float(); ox = f.x; oy = f.y; }
    const float W = (float)(P.imax[0] - P.imin[0]), H = (float)(P.imax[1] - P.imin[1]);
    const float uvx = ((float)px + ox - P.imin[0]) / W, uvy = ((float)py + oy - P.imin[1]) / H;
    const float cx = 2.f * uvx - 1.f, cy = -(2.f * uvy - 1.f);
    const float sx = P.proj[0], sy = P.proj[1], offx = P.proj[2], offy = P.proj[3], nr = P.proj[4];
    float3 ld;
    if (P.proj[7] < 0.f) ld = f3((cx - offx) / sx, (cy - offy) / sy, nr);
    else {
        const float sg = nr > 0.f ? 1.f : (nr < 0.f ? -1.f : 0.f);
        ld = f3(nr * (cx * sg - offx) / sx, nr * (cy * sg - offy) / sy, nr);
    }
    ld = normalize(ld);
    const float* c = P.cam;
    const float3 wd = normalize(f3(c[0] * ld.x + c[1] * ld.y + c[2] * ld.z, c[4] * ld.x + c[5] * ld.y + c[6] * ld.z,
                                   c[8] * ld.x + c[9] * ld.y + c[10] * ld.z));
    const float3 d = unpack_normal(pack_normal(wd));
    uint32_t meta = (sample == 0 ? 0x100u : 0u);  // path length 0; bit 8: write AOVs
    if (P.cache_on && pcg_hash(slot ^ pcg_hash(P.frame_seed + sample)) % P.train_mod == 0u) meta |= 0x200u;  // training path
    const PathQueue& q = P.q[0];
    q.s0[i] = make_float4(c[3], c[7], c[11], 0.f);
    q.s1[i] = make_float4(d.x, d.y, d.z, 1.f);
    q.s2[i] = make_float4(1.f, 1.f, __uint_as_float(slot), __uint_as_float(meta));
    q.s3[i] = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
}

// ---------------------------------------------------------------- per-bounce bookkeeping
// Counters before a bounce.  The previous bounce's shadow rays are retired into the statistics:
// already traced, or (sh_merge) about to be traced by this bounce's k_trace from their own count,
// while this bounce's shade appends to the other one.
__global__ void k_bounce_setup(PTParams P, uint32_t parity, int first) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t cur = sh_counter(P), prev = P.sh_merge ? (cur == C_SHADOW ? C_SHADOW1 : C_SHADOW) : cur;
    if (!first) P.stats[S_SHADOW] += P.counters[prev];
    P.stats[S_EXT] += P.counters[parity];
    P.counters[1 - parity] = 0;
    P.counters[cur] = 0;
    P.counters[C_WORK_EXT] = 0;
    P.counters[C_WORK_OCC] = 0;
    P.counters[C_CACHEQ] = 0;
}
// Before the trailing k_occlude of a wave whose shadow tracing was merged into k_trace.
__global__ void k_occlude_setup(PTParams P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    P.counters[C_WORK_OCC] = 0;
}
__global__ void k_wave_finish(PTParams P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    P.stats[S_SHADOW] += P.counters[sh_counter(P)];
    P.counters[C_SHADOW] = 0;
    P.counters[C_SHADOW1] = 0;
}

// ---------------------------------------------------------------- batched streaming mode
// Path regeneration: before every bounce the queue is topped up to capacity with new camera paths
// (taken in path-id order across all views), so every launch works on a full queue however
// unevenly Russian roulette and escapes shorten the paths.
__global__ void k_stream_setup(PTParams P, uint32_t parity, int first) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long* ss = P.stream_state;
    // the previous iteration's shadow rays are retired as in k_bounce_setup
    const uint32_t cur = sh_counter(P), prev = P.sh_merge ? (cur == C_SHADOW ? C_SHADOW1 : C_SHADOW) : cur;
    if (!first) P.stats[S_SHADOW] += P.counters[prev];
    const uint32_t live = P.counters[parity];
    const unsigned long long left = P.total_paths - ss[0];
    const uint32_t fill = (uint32_t)min((unsigned long long)(P.capacity - live), left);
    ss[1] = ss[0];
    ss[2] = fill;
    ss[0] += fill;
    ss[3] = (live + fill == 0) ? 1ull : 0ull;
    P.counters[parity] = live + fill;
    P.stats[S_EXT] += live + fill;
    P.counters[1 - parity] = 0;
    P.counters[cur] = 0;
    P.counters[C_WORK_EXT] = 0;
    P.counters[C_WORK_OCC] = 0;
    P.counters[C_CACHEQ] = 0;
}

// New camera paths for path ids [base, base + fill), appended after the live paths.
S2D void regen_one(const PTParams& P, uint32_t parity, uint32_t fill, uint32_t i) {
    const unsigned long long id = P.stream_state[1] + i;
    const uint32_t q = P.counters[parity] - fill + i;
    const PathQueue& Q = P.q[parity];
    if (id >= P.image_paths) {
        // radiance-cache training path: a seeded pixel of the batch, its own sample seed, slot =
        // its training accumulator (bit 31), meta bit 9 (runs to its end and records its vertices)
        const uint32_t ti = (uint32_t)(id - P.image_paths);
        const uint32_t g = pcg_hash(ti ^ pcg_hash(P.frame_seed ^ 0x9e3779b9u)) % P.batch_pixels;
        uint32_t v = 0;
        while (v + 1 < P.nviews && P.views[v + 1].pixel_offset <= g) ++v;
        const ViewEntry& V = P.views[v];
        const uint32_t pix = g - V.pixel_offset, px = pix % V.width, py = pix / V.width;
        Rng rng = make_rng(px, py, P.frame_seed + P.view_spp + ti, (P.flags & S2F_PCG32) != 0);
        float ox = 0.5f, oy = 0.5f;
        if (P.flags & S2F_JITTER) { const float4 f = rng.next_float(); ox = f.x; oy = f.y; }
        const float3 d = camera_dir(V.proj, V.imin, V.imax, V.cam, px, py, ox, oy);
        Q.s0[q] = make_float4(V.cam[3], V.cam[7], V.cam[11], 0.f);
        Q.s1[q] = make_float4(d.x, d.y, d.z, 1.f);
        Q.s2[q] = make_float4(1.f, 1.f, __uint_as_float(kTrainSlot | ti), __uint_as_float(0x200u | (v << 16)));
        Q.s3[q] = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
        return;
    }
    uint32_t v = 0;
    while (v + 1 < P.nviews && P.views[v + 1].path_offset <= id) ++v;
    const ViewEntry& V = P.views[v];
    const unsigned long long local = id - V.path_offset;
    // path order inside a view: pixel (row-major), then sample (as k_raygen): a warp takes the
    // samples of one or a few neighbouring pixels, whose camera rays traverse nearly the same nodes
    const uint32_t pix = (uint32_t)(local / P.view_spp);
    const uint32_t sample = (uint32_t)(local - (unsigned long long)pix * P.view_spp);
    const uint32_t py = pix / V.width, px = pix - py * V.width;
    Rng rng = make_rng(px, py, P.frame_seed + sample, (P.flags & S2F_PCG32) != 0);
    float ox = 0.5f, oy = 0.5f;
    if (P.flags & S2F_JITTER) { const float4 f = rng.next_float(); ox = f.x; oy = f.y; }
    const float3 d = camera_dir(V.proj, V.imin, V.imax, V.cam, px, py, ox, oy);
    // meta: path length 0, bit 8 = write AOVs, bits 16..23 = view
    const uint32_t meta = (sample == 0 ? 0x100u : 0u) | (v << 16);
    Q.s0[q] = make_float4(V.cam[3], V.cam[7], V.cam[11], 0.f);
    Q.s1[q] = make_float4(d.x, d.y, d.z, 1.f);
    Q.s2[q] = make_float4(1.f, 1.f, __uint_as_float(V.pixel_offset + pix), __uint_as_float(meta));
    Q.s3[q] = make_uint4(rng.px, rng.py, rng.seed, rng.ctr);
}

__global__ void k_regen(PTParams P, uint32_t parity) {
    const uint32_t fill = (uint32_t)P.stream_state[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < fill; i += gridDim.x * blockDim.x)
        regen_one(P, parity, fill, i);
}

// Fixed-point totals -> mean radiance * 2^exposure for one view.
__global__ void k_resolve_fx(const unsigned long long* __restrict__ total_fx, uint32_t pixel_offset, uint32_t pixels,
                             float scale, float4* __restrict__ out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const unsigned long long* t = total_fx + 4 * (size_t)(pixel_offset + p);
    const float s = scale / S2_FX_SCALE;
    out[p] = make_float4((float)((double)t[0] * s), (float)((double)t[1] * s), (float)((double)t[2] * s), 1.f);
}

// ---------------------------------------------------------------- extend / occlude
// Persistent traversal with lane refill: every lane owns one ray at a time and advances it one
// node per loop iteration; when at least kRefillMin lanes of a warp have finished their rays (or
// all have), the warp fetches that many new rays from the global work counter with one atomic.
// Lanes therefore stay busy while long rays finish, instead of the whole warp waiting for its
// slowest ray (dynamic ray fetch in the manner of Aila and Laine, HPG 2009).
constexpr uint32_t kRefillMin = 8;  // default of PTParams::refill_min
constexpr uint32_t kNoRay = 0xffffffffu;

// Warp-sum of the fetch counters, one 64-bit atomic per warp (counting runs only).
S2D void add_fetches(unsigned long long* stats, uint32_t node_stat, const TravCounters& c) {
    uint32_t n = c.nodes, t = c.tris;
    for (int o = 16; o > 0; o >>= 1) { n += __shfl_xor_sync(0xffffffffu, n, o); t += __shfl_xor_sync(0xffffffffu, t, o); }
    if ((threadIdx.x & 31u) == 0) { atomicAdd(&stats[node_stat], (unsigned long long)n); atomicAdd(&stats[node_stat + 1], (unsigned long long)t); }
}

// Gives idle lanes new work items [0, count) from `work`; returns the lane's item or kNoRay.
S2D uint32_t refill(uint32_t* work, uint32_t count, uint32_t item, bool& exhausted, uint32_t refill_min) {
    const bool need = item == kNoRay && !exhausted;
    const uint32_t needm = __ballot_sync(0xffffffffu, need);
    const uint32_t activem = __ballot_sync(0xffffffffu, item != kNoRay);
    if (needm && ((uint32_t)__popc(needm) >= (refill_min ? refill_min : kRefillMin) || activem == 0)) {
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t leader = __ffs(needm) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(work, (uint32_t)__popc(needm));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (need) {
            const uint32_t idx = base + __popc(needm & ((1u << lane) - 1u));
            if (idx < count) item = idx;
            else exhausted = true;
        }
    }
    return item;
}

// Closest hit of the live path queue.  Hit record: {t, triangle record index, b1, b2}.
// `stack`: the block's shared-memory traversal stacks (S2_STACK_SMEM entries per thread).
template <bool COUNT>
S2D void extend_queue(const PTParams& P, uint32_t parity, uint2* stack) {
    uint2 lstack[S2_STACK_DEPTH - S2_STACK_SMEM];
    const uint32_t count = P.counters[parity];
    const PathQueue q = P.q[parity];
    TravCounters c{0, 0};
    TravRay r;
    TravState st;
    TravHit h;
    uint32_t ray = kNoRay;
    bool exhausted = false;
    while (true) {
        const uint32_t prev = ray;
        ray = refill(&P.counters[C_WORK_EXT], count, ray, exhausted, P.refill_min);
        if (!__any_sync(0xffffffffu, ray != kNoRay)) break;
        if (ray != kNoRay && prev == kNoRay) {
            if (P.ray_sorted) ray = P.sort_perm[ray];  // coherence order; results stay per queue slot
            const float4 a = q.s0[ray], b = q.s1[ray];
            r = make_trav_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), 0.f);
            trav_begin(st, h, S2_INF);
            if (P.hint_tri) {
                // the pixel centre's triangle as a first candidate: a hit there becomes the closest
                // hit so far, exactly as if the traversal had found it first (hits are resolved by
                // distance, then by the lowest instance and primitive, in any visiting order)
                const uint32_t ti = P.hint_tri[__float_as_uint(q.s2[ray].z) % P.pixels];
                if (ti != 0xffffffffu) {
                    const float4 t0 = __ldg(P.scene.tris + 3 * (size_t)ti), t1 = __ldg(P.scene.tris + 3 * (size_t)ti + 1);
                    const float4 t2 = __ldg(P.scene.tris + 3 * (size_t)ti + 2);
                    float t, b1, b2;
                    if (COUNT) c.tris++;
                    if (!(__float_as_uint(t2.w) & S2_TRI_ALPHA_TESTED) &&
                        intersect_triangle(r, ld3(t0), ld3(t1), ld3(t2), h.t, t, b1, b2)) {
                        h.t = t; h.tri = ti; h.instance = __float_as_uint(t0.w); h.primitive = __float_as_uint(t1.w);
                        h.b1 = b1; h.b2 = b2;
                    }
                }
            }
        }
        // counting runs take the sequential nearest-first walk, the order the CPU BVH8 walker
        // restates.  The postponed-triangle order visits the same nodes: a lane tests its pending
        // triangles before its next box test, and the next node is chosen from box tests alone.
        const bool tri_step = COUNT ? false : trav_vote_tri(ray != kNoRay, st, P.trav.vote8);
        if (ray != kNoRay) {
            const SceneAlphaTest alpha{&P.scene, !(P.flags & S2F_NO_ALPHA)};
            if (COUNT ? trav_step<false, true>(r, st, P.scene.nodes, P.scene.tris, stack + threadIdx.x, kTravBlock, lstack, h, c, alpha)
                      : trav_step_pp<false, false>(r, st, P.scene.nodes, P.scene.tris, stack + threadIdx.x, kTravBlock, lstack, h, c,
                                                   tri_step, P.trav.tris_per_step, alpha)) {
                if (!st.ok) atomicOr(P.status, 1);
                P.hits[ray] = make_float4(h.t, __uint_as_float(h.tri), h.b1, h.b2);
                if (P.sort_on)  // key: the instance's material word (material address | instance type), misses last
                    P.sort_keys[ray] = h.tri == 0xffffffffu ? kSortBuckets - 1u : P.scene.instances[h.instance].x % (kSortBuckets - 1u);
                ray = kNoRay;
            }
        }
    }
    if (COUNT) add_fetches(P.stats, S_EXT_NODES, c);
}

template <bool COUNT>
__global__ void __launch_bounds__(kTravBlock) k_extend(const __grid_constant__ PTParams P, uint32_t parity) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTravBlock];
    extend_queue<COUNT>(P, parity, stack);
}

// The closest-hit triangle record (or none) of every pixel's centre ray, for the camera launch's
// first candidate.  One thread per pixel.
__global__ void __launch_bounds__(kTravBlock) k_pixel_hint(const __grid_constant__ PTParams P, uint32_t* __restrict__ hint) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTravBlock];
    const uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= P.pixels) return;
    const uint32_t px = pix % P.width, py = pix / P.width;
    const float3 d = camera_dir(P.proj, P.imin, P.imax, P.cam, px, py, 0.5f, 0.5f);
    TravHit h;
    TravCounters c{0, 0};
    const SceneAlphaTest alpha{&P.scene, !(P.flags & S2F_NO_ALPHA)};
    traverse<false, false>(make_trav_ray(f3(P.cam[3], P.cam[7], P.cam[11]), d, 0.f), S2_INF, P.scene.nodes, P.scene.tris,
                           stack + threadIdx.x, kTravBlock, h, c, alpha);
    hint[pix] = h.tri;
}

// The persistent any-hit loop over the shadow queue (sh_o: origin + t_max, sh_d: direction): warps
// refill lanes from the work counter; `on_visible(ray)` runs for every unoccluded ray.
// `count_idx`: the counter holding the queue's length; `stack` as in extend_queue.
template <bool COUNT, class OnVisible>
S2D void occlude_queue(const PTParams& P, uint32_t count_idx, uint2* stack, const OnVisible& on_visible) {
    uint2 lstack[S2_STACK_DEPTH - S2_STACK_SMEM];
    const uint32_t count = P.counters[count_idx];
    TravCounters c{0, 0};
    TravRay r;
    TravState st;
    TravHit h;
    uint32_t ray = kNoRay;
    bool exhausted = false;
    while (true) {
        const uint32_t prev = ray;
        ray = refill(&P.counters[C_WORK_OCC], count, ray, exhausted, P.refill_min);
        if (!__any_sync(0xffffffffu, ray != kNoRay)) break;
        if (ray != kNoRay && prev == kNoRay) {
            const float4 o = P.sh_o[ray], d = P.sh_d[ray];
            r = make_trav_ray(f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), 0.f);
            trav_begin(st, h, o.w);
        }
        const bool tri_step = COUNT ? false : trav_vote_tri(ray != kNoRay, st, P.trav.vote8);
        if (ray != kNoRay) {
            const SceneAlphaTest alpha{&P.scene, !(P.flags & S2F_NO_ALPHA)};
            if (COUNT ? trav_step<true, true>(r, st, P.scene.nodes, P.scene.tris, stack + threadIdx.x, kTravBlock, lstack, h, c, alpha)
                      : trav_step_pp<true, false>(r, st, P.scene.nodes, P.scene.tris, stack + threadIdx.x, kTravBlock, lstack, h, c,
                                                  tri_step, P.trav.tris_per_step, alpha)) {
                if (!st.ok) atomicOr(P.status, 1);
                if (h.tri == 0xffffffffu) on_visible(ray);
                ray = kNoRay;
            }
        }
    }
    if (COUNT) add_fetches(P.stats, S_SH_NODES, c);
}

// ProcessShadowRays (testrenderer.slang:1147-1166) without the fixed-point atomics: each shadow
// ray belongs to one accumulator slot (sh_d.w) and adds its contribution (sh_c) when unoccluded.
template <bool COUNT>
__global__ void __launch_bounds__(kTravBlock) k_occlude(const __grid_constant__ PTParams P) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTravBlock];
    occlude_queue<COUNT>(P, sh_counter(P), stack, [&](uint32_t ray) {
        const float4 cc = P.sh_c[ray];
        add_contrib(P, __float_as_uint(P.sh_d[ray].w), f3(cc.x, cc.y, cc.z));
    });
}

// One bounce's closest hits followed by the previous bounce's shadow rays (count in counter
// `sh_prev`), in one persistent launch: a warp whose extension work has run out takes shadow rays
// while other warps finish their long extension rays, so the two launches' tails overlap.  The
// contributions reach the accumulators before the next shade, as with a separate k_occlude.
template <bool COUNT>
__global__ void __launch_bounds__(kTravBlock, 9) k_trace(const __grid_constant__ PTParams P, uint32_t parity, uint32_t sh_prev) {
    __shared__ uint2 stack[S2_STACK_SMEM * kTravBlock];
    extend_queue<COUNT>(P, parity, stack);
    occlude_queue<COUNT>(P, sh_prev, stack, [&](uint32_t ray) {
        const float4 cc = P.sh_c[ray];
        add_contrib(P, __float_as_uint(P.sh_d[ray].w), f3(cc.x, cc.y, cc.z));
    });
}

// ---------------------------------------------------------------- accumulation
// Sum the wave's per-sample slots into the per-pixel total in a fixed order (sample 0 first) and
// clear them.  Loads are issued eight samples at a time so each thread keeps eight 16-byte reads
// in flight; the additions stay in sample order, so the sums do not depend on the batching.
__global__ void k_reduce(PTParams P, float4* __restrict__ total) {
    constexpr uint32_t kBatch = 8;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.pixels) return;
    float4 t = total[p];
    const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t k0 = 0; k0 < P.wave_samples; k0 += kBatch) {
        float4 a[kBatch];
#pragma unroll
        for (uint32_t j = 0; j < kBatch; ++j)
            a[j] = k0 + j < P.wave_samples ? __ldcs(P.accum + (size_t)(k0 + j) * P.pixels + p) : zero;
#pragma unroll
        for (uint32_t j = 0; j < kBatch; ++j) {
            if (k0 + j < P.wave_samples) {
                t.x += a[j].x; t.y += a[j].y; t.z += a[j].z;
                P.accum[(size_t)(k0 + j) * P.pixels + p] = zero;
            }
        }
    }
    total[p] = t;
}

// Mean over samples times 2^exposure (tonemap.slang:154), alpha 1.
__global__ void k_resolve(const float4* __restrict__ total, uint32_t pixels, float inv_spp, float exposure_scale,
                          float4* __restrict__ out) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= pixels) return;
    const float4 t = total[p];
    const float s = inv_spp * exposure_scale;
    out[p] = make_float4(t.x * s, t.y * s, t.z * s, 1.f);
}

}  // namespace s2

namespace s2 {
// Radiance-cache training targets: the radiance a training path gathered after each recorded vertex
// (its final accumulator minus the value when the vertex was reached), per unit throughput.
__global__ void k_cache_targets(PTParams P) {
    const uint32_t n = min(P.counters[C_TRAIN], P.tr_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t slot = __float_as_uint(P.tr_pos[i].w) & ~kTrainSlot;
        const float4 fin = P.accum[slot], r0 = P.tr_rad[i], t = P.tr_thr[i];
        const float tx = t.x > 1e-8f ? (fin.x - r0.x) / t.x : 0.f;
        const float ty = t.y > 1e-8f ? (fin.y - r0.y) / t.y : 0.f;
        const float tz = t.z > 1e-8f ? (fin.z - r0.z) / t.z : 0.f;
        P.tr_rad[i] = make_float4(fmaxf(tx, 0.f), fmaxf(ty, 0.f), fmaxf(tz, 0.f), 0.f);
    }
}
}  // namespace s2

namespace s2 {
// ---------------------------------------------------------------- material-key counting sort
// Histogram of the live queue's keys: per-block shared histogram with one shared atomic per group
// of equal keys in a warp (queues are spatially coherent, so most lanes of a warp share a key),
// then one global atomic per non-empty bucket and block.
__global__ void __launch_bounds__(256) k_sort_hist(PTParams P, uint32_t parity) {
    __shared__ uint32_t h[kSortBuckets];
    for (uint32_t b = threadIdx.x; b < kSortBuckets; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint32_t n = P.counters[parity];
    const uint32_t rounded = (n + 31u) & ~31u;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < rounded; i += gridDim.x * blockDim.x) {
        const bool live = i < n;
        const uint32_t key = live ? P.sort_keys[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (live && lane == (uint32_t)__ffs(peers) - 1u) atomicAdd(&h[key], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < kSortBuckets; b += blockDim.x)
        if (h[b]) atomicAdd(&P.sort_hist[b], h[b]);
}

// Exclusive scan of the histogram in place (one block of 1024 threads, four buckets each).
__global__ void __launch_bounds__(1024) k_sort_scan(PTParams P) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    uint32_t v[4], sum = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) { v[k] = P.sort_hist[4 * t + k]; sum += v[k]; }
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        const uint32_t x = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
#pragma unroll
    for (int k = 0; k < 4; ++k) { P.sort_hist[4 * t + k] = run; run += v[k]; }
}

// Scatter: sort_perm[offset[key] + rank] = i.  Each block takes one contiguous chunk of the
// queue: it counts its keys in shared memory, reserves its range of every non-empty bucket with
// one global atomic, and ranks its items inside those ranges with shared atomics (one per group of
// equal keys in a warp).  The order inside a bucket is not fixed; shading results do not depend on
// it (every path keeps its own random state and accumulator slot).
__global__ void __launch_bounds__(256) k_sort_scatter(PTParams P, uint32_t parity) {
    __shared__ uint32_t h[kSortBuckets];
    for (uint32_t b = threadIdx.x; b < kSortBuckets; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint32_t n = P.counters[parity];
    const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 255u) & ~255u;
    const uint32_t begin = min(n, blockIdx.x * chunk), end = min(n, begin + chunk);
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = begin + threadIdx.x; i < begin + chunk; i += blockDim.x) {  // warp-uniform trip count
        const bool live = i < end;
        const uint32_t key = live ? P.sort_keys[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (live && lane == (uint32_t)__ffs(peers) - 1u) atomicAdd(&h[key], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < kSortBuckets; b += blockDim.x)
        if (h[b]) h[b] = atomicAdd(&P.sort_hist[b], h[b]);
    __syncthreads();
    for (uint32_t i = begin + threadIdx.x; i < begin + chunk; i += blockDim.x) {
        const bool live = i < end;
        const uint32_t key = live ? P.sort_keys[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = __ffs(peers) - 1u;
        uint32_t base = 0;
        if (live && lane == leader) base = atomicAdd(&h[key], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (live) P.sort_perm[base + __popc(peers & ((1u << lane) - 1u))] = i;
    }
}
}  // namespace s2
