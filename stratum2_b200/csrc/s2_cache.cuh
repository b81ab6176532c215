// Learned radiance cache (no counterpart in the reference): a multiresolution hash-grid encoding of
// the world-space position (16 levels x 2 f16 features, 2^19 entries per level, resolutions
// geometric from 16 to 2048 over the cache's box; the published Instant-NGP encoding, Mueller et
// al. 2022) feeding a 32 -> 64 -> 64 -> 3 ReLU MLP without biases (6,336 weights), evaluated with
// f16 operands and f32 accumulation on the tensor cores (tcgen05, accumulators in TMEM).
//
// Per CTA of 128 threads and per tile of 128 queries, thread t owns query row t: it writes the
// row's 32 encoded features into a K-major shared-memory tile, one thread issues the MMAs of a
// layer, everybody waits on an mbarrier, reads its TMEM lane (row t), applies ReLU and writes the
// next layer's input row.  The weights are staged in shared memory once per CTA.
#pragma once
#include <cuda_fp16.h>

#include "s2_math.cuh"
#include "s2_tc.cuh"

namespace s2 {

constexpr uint32_t kCacheLevels = 16;
constexpr uint32_t kCacheFeatures = 2;
constexpr uint32_t kCacheIn = kCacheLevels * kCacheFeatures;  // 32
constexpr uint32_t kCacheHidden = 64;
constexpr uint32_t kCacheOut = 3;
constexpr uint32_t kCacheOutPad = 16;  // N of the last MMA
constexpr uint32_t kCacheW1 = kCacheHidden * kCacheIn;       // 2048
constexpr uint32_t kCacheW2 = kCacheHidden * kCacheHidden;   // 4096
constexpr uint32_t kCacheW3 = kCacheOut * kCacheHidden;      // 192
constexpr uint32_t kCacheWeights = kCacheW1 + kCacheW2 + kCacheW3;  // 6336
constexpr uint32_t kCacheTile = 128;

// Byte images of the weights in the shared-memory operand layout (K-major core matrices):
// W1 64 x 32, W2 64 x 64, W3 padded to 16 x 64 (rows 3..15 zero).
constexpr uint32_t kW1Bytes = kCacheHidden * kCacheIn * 2;      // 4096
constexpr uint32_t kW2Bytes = kCacheHidden * kCacheHidden * 2;  // 8192
constexpr uint32_t kW3Bytes = kCacheOutPad * kCacheHidden * 2;  // 2048
constexpr uint32_t kWImageBytes = kW1Bytes + kW2Bytes + kW3Bytes;
// Transposed copies for the backward pass (B operands of dH1 = dH2 W2 and dX = dH1 W1):
// W2T 64 x 64 with element (i, o) = W2[o][i], W1T 32 x 64 with element (i, o) = W1[o][i].
constexpr uint32_t kW2TBytes = kCacheHidden * kCacheHidden * 2;  // 8192
constexpr uint32_t kW1TBytes = kCacheIn * kCacheHidden * 2;      // 4096
constexpr uint32_t kWImageTrainBytes = kWImageBytes + kW2TBytes + kW1TBytes;
// Backward activations are scaled by this power of two before their f16 rounding (keeps them in
// range), and unscaled in f32 when gradients leave the tensor cores.
constexpr float kCacheGradScale = 1.f / 64.f;

struct CacheDev {
    const __half2* table;        // [levels][2^log2_table] feature pairs
    uint32_t log2_table;
    float res[kCacheLevels];     // grid resolution per level
    uint32_t dense[kCacheLevels];// 1: level indexed densely (all its bricks fit the table)
    uint32_t nbrick[kCacheLevels];// bricks per axis of a dense level: ceil((res + 1) / 2)
    float3 box_min, box_inv_extent;
    const uint4* wimage;         // kWImageTrainBytes: W1, W2, W3 (padded), W2T, W1T in operand layout
    int* status;                 // bit 2: a tensor-core wait timed out
    // failure-detection test (s2_inject_wait_timeout): nonzero makes the inference kernel wait on
    // its first-layer barrier without issuing that layer's MMA or commit -- an arrival that never
    // comes -- polling at most this many times in each of its waits; 0 = off
    uint32_t wait_test;
    // training
    float* grad_w;               // summed per-record gradients of the weights
    float* grad_t;               // summed per-record gradients of the table, [levels][entries][2]
    float* loss_sum;             // summed per-record losses
};

// Normalised position in [0, 1) of the cache box.
S2D float3 cache_unit(const CacheDev& c, float3 p) {
    float3 u = (p - c.box_min) * c.box_inv_extent;
    const float hi = 0.99999994f;
    u.x = fminf(fmaxf(u.x, 0.f), hi);
    u.y = fminf(fmaxf(u.y, 0.f), hi);
    u.z = fminf(fmaxf(u.z, 0.f), hi);
    return u;
}

// Table layout: the grid vertices of a level are grouped in 2 x 2 x 2 bricks of 8 consecutive
// entries (32 bytes, one L2 sector), so the 8 corners of a cell touch 1 to 8 sectors (3.375 on
// average) instead of 8.  Bricks are placed densely when they all fit the level's table, else by
// the spatial hash of Instant-NGP (Mueller et al. 2022) applied to the brick coordinates.
S2D uint32_t cache_index(const CacheDev& c, uint32_t level, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t mask = (1u << (c.log2_table - 3u)) - 1u;
    const uint32_t bx = x >> 1, by = y >> 1, bz = z >> 1;
    uint32_t b;
    if (c.dense[level]) {
        const uint32_t n = c.nbrick[level];
        b = (bx + n * (by + n * bz)) & mask;
    } else {
        b = (bx ^ (by * 2654435761u) ^ (bz * 805459861u)) & mask;
    }
    return (b << 3) | (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
}

// The 32 encoded features of one position (trilinear interpolation of the 8 corner entries per
// level), as 16 half2 values (level l in out[l]).
S2D void cache_encode(const CacheDev& c, float3 p, __half2 out[kCacheLevels]) {
    const float3 u = cache_unit(c, p);
#pragma unroll 4
    for (uint32_t l = 0; l < kCacheLevels; ++l) {
        const float r = c.res[l];
        const float fx = u.x * r, fy = u.y * r, fz = u.z * r;
        const float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
        const float wx = fx - ix, wy = fy - iy, wz = fz - iz;
        const uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
        const __half2* tab = c.table + ((size_t)l << c.log2_table);
        float a0 = 0.f, a1 = 0.f;
#pragma unroll
        for (uint32_t k = 0; k < 8; ++k) {
            const uint32_t dx = k & 1u, dy = (k >> 1) & 1u, dz = k >> 2;
            const float w = (dx ? wx : 1.f - wx) * (dy ? wy : 1.f - wy) * (dz ? wz : 1.f - wz);
            const float2 f = __half22float2(__ldg(tab + cache_index(c, l, x0 + dx, y0 + dy, z0 + dz)));
            a0 += w * f.x;
            a1 += w * f.y;
        }
        out[l] = __floats2half2_rn(a0, a1);
    }
}

// One corner entry (f16x2 bits) of a 16-byte quad: the 2 x 2 entries of one z layer of a brick.
S2D uint32_t cache_quad_entry(uint4 q, uint32_t xb, uint32_t yb) {
    const uint32_t lo = xb ? q.y : q.x, hi = xb ? q.w : q.z;
    return yb ? hi : lo;
}

// Levels l0 .. l0+3 of the encoding of one position: the values of cache_encode, gathered by quads.
// A z layer of the cell's 2 x 2 x 2 corners lies in 1, 2 or 4 quads (whether x0 and y0 are odd),
// so a level issues 4.5 16-byte loads on average instead of eight 4-byte ones; the corners are
// picked from the quads by selects and summed in cache_encode's order.
S2D void cache_encode4(const CacheDev& c, float3 p, uint32_t l0, __half2 out[4]) {
    const float3 u = cache_unit(c, p);
    const uint32_t mask = (1u << (c.log2_table - 3u)) - 1u;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t l = l0 + j;
        const float r = c.res[l];
        const float fx = u.x * r, fy = u.y * r, fz = u.z * r;
        const float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
        const float wx = fx - ix, wy = fy - iy, wz = fz - iz;
        const uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
        const uint32_t ox = x0 & 1u, oy = y0 & 1u, oz = z0 & 1u;
        const uint32_t bx = x0 >> 1, by = y0 >> 1, bz = z0 >> 1;
        const uint4* tq = (const uint4*)(c.table + ((size_t)l << c.log2_table));
        // brick index = combine(x term, y term, z term) & mask, as in cache_index
        const bool dense = c.dense[l] != 0;
        const uint32_t n = c.nbrick[l];
        const uint32_t tx0 = bx, tx1 = bx + ox;
        const uint32_t ty0 = dense ? n * by : by * 2654435761u, ty1 = dense ? n * (by + oy) : (by + oy) * 2654435761u;
        const uint32_t tz0 = dense ? n * n * bz : bz * 805459861u, tz1 = dense ? n * n * (bz + oz) : (bz + oz) * 805459861u;
        float a0 = 0.f, a1 = 0.f;
#pragma unroll
        for (uint32_t dz = 0; dz < 2; ++dz) {
            const uint32_t tz = dz ? tz1 : tz0, zb = oz ^ dz;
            const uint32_t b00 = (dense ? tx0 + ty0 + tz : tx0 ^ ty0 ^ tz) & mask;
            const uint32_t b10 = (dense ? tx1 + ty0 + tz : tx1 ^ ty0 ^ tz) & mask;
            const uint32_t b01 = (dense ? tx0 + ty1 + tz : tx0 ^ ty1 ^ tz) & mask;
            const uint32_t b11 = (dense ? tx1 + ty1 + tz : tx1 ^ ty1 ^ tz) & mask;
            const uint4 q00 = __ldg(tq + ((b00 << 1) | zb));
            uint4 q10 = q00, q01 = q00, q11 = q00;
            if (ox) q10 = __ldg(tq + ((b10 << 1) | zb));
            if (oy) q01 = __ldg(tq + ((b01 << 1) | zb));
            if (ox & oy) q11 = __ldg(tq + ((b11 << 1) | zb));
            else q11 = ox ? q10 : q01;
            const float wz_ = dz ? wz : 1.f - wz;
#pragma unroll
            for (uint32_t k = 0; k < 4; ++k) {
                const uint32_t dx = k & 1u, dy = k >> 1;
                const uint4 q = dx ? (dy ? q11 : q10) : (dy ? q01 : q00);
                const uint32_t h = cache_quad_entry(q, ox ^ dx, oy ^ dy);
                const float w = (dx ? wx : 1.f - wx) * (dy ? wy : 1.f - wy) * wz_;
                __half2 hv;
                *(uint32_t*)&hv = h;
                const float2 f = __half22float2(hv);
                a0 += w * f.x;
                a1 += w * f.y;
            }
        }
        out[j] = __floats2half2_rn(a0, a1);
    }
}

S2D void block_sync_tc() {
    fence_smem_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
}

// Shared-memory plan of the inference kernel (bytes): weights, input tile, hidden tile.
constexpr uint32_t kInfSmemW = 0;
constexpr uint32_t kInfSmemX = kWImageBytes;                         // 128 x 32 f16
constexpr uint32_t kInfSmemH = kInfSmemX + kCacheTile * kCacheIn * 2; // 128 x 64 f16
constexpr uint32_t kInfSmemBytes = kInfSmemH + kCacheTile * kCacheHidden * 2;
// Inference CTA: 256 threads; two threads encode one query (eight levels = two 16-byte operand
// chunks each), the first warpgroup runs the MLP.  Two CTAs per SM: the MLP chain of one (three
// dependent MMAs, 12 of 16 warps idle) overlaps the table gathers of the other.
constexpr uint32_t kInfThreads = 256;
constexpr uint32_t kInfCtasPerSm = 2;
constexpr uint32_t kInfParts = kInfThreads / kCacheTile;  // threads per query
static_assert(kInfParts * kCacheTile == kInfThreads && 4 % kInfParts == 0, "whole operand chunks per thread");

// Writes 8 f16 values (one 16-byte chunk) of row r, chunk q of a K-major tile.
S2D void store_chunk(uint8_t* tile, uint32_t r, uint32_t q, uint32_t K, const __half2 h[4]) {
    uint4 v;
    v.x = *(const uint32_t*)&h[0];
    v.y = *(const uint32_t*)&h[1];
    v.z = *(const uint32_t*)&h[2];
    v.w = *(const uint32_t*)&h[3];
    *(uint4*)(tile + kmaj_offset(r, q * 8u, K)) = v;
}

// Reads 64 accumulator columns at TMEM column `col` of this thread's lane, applies ReLU and writes
// them as row `row` of the K=64 tile `dst`.
S2D void tmem_relu_to_tile(uint32_t tlane, uint32_t col, uint8_t* dst, uint32_t row) {
#pragma unroll
    for (uint32_t g = 0; g < 4; ++g) {
        float v[16];
        tmem_ld16(tlane + col + 16u * g, v);
        __half2 h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = __floats2half2_rn(fmaxf(v[2 * i], 0.f), fmaxf(v[2 * i + 1], 0.f));
        store_chunk(dst, row, 2u * g, kCacheHidden, h);
        store_chunk(dst, row, 2u * g + 1u, kCacheHidden, h + 4);
    }
}

// Radiance cache inference: out[i] = MLP(encode(pos[i])), raw (unclamped) outputs.  With `tput`
// (the path tracer's terminal vertices) the result is instead added to the path's accumulator:
// accum[slot] += tput[i] * max(y, 0), slot in pos[i].w, or with `total_fx` (the batched renderer)
// to the pixel's fixed-point totals.  n_dev (optional) caps n with a device count.
// Persistent: grid-stride over tiles of 128 queries; kInfThreads threads; kInfSmemBytes dynamic smem.
__global__ void __launch_bounds__(kInfThreads, kInfCtasPerSm) k_cache_infer(const __grid_constant__ CacheDev c, const float4* __restrict__ pos,
                                                                uint32_t n, const uint32_t* __restrict__ n_dev,
                                                                float4* __restrict__ out, const float4* __restrict__ tput,
                                                                float4* __restrict__ accum,
                                                                unsigned long long* __restrict__ total_fx) {
    if (n_dev) n = min(n, *n_dev);
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const bool mlp = warp < 4;  // the warpgroup whose lanes are the tile's rows
    for (uint32_t i = t; i < kWImageBytes / 16; i += kInfThreads) ((uint4*)(smem + kInfSmemW))[i] = c.wimage[i];
    if (warp == 0) {
        tmem_alloc(&tmem_base, 128);
        tmem_relinquish();
    }
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    fence_smem_async();
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t tlane = tmem + ((32u * (warp & 3u)) << 16);  // this warp's lane quarter
    const uint32_t s_w1 = smem_addr(smem + kInfSmemW), s_w2 = s_w1 + kW1Bytes, s_w3 = s_w2 + kW2Bytes;
    const uint32_t s_x = smem_addr(smem + kInfSmemX), s_h = smem_addr(smem + kInfSmemH);
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t wait_limit = c.wait_test ? c.wait_test : kMbarWaitLimit;
    // MMA completion for the MLP warps (the others only take part in the block barriers)
    auto done = [&](bool issued) {
        if (!mlp) return;
        const bool w = ok && issued && mbar_wait(&bar, phase, wait_limit);
        if (w) phase ^= 1u;
        ok = __all_sync(0xffffffffu, w);
    };
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        {
            // encode: thread t takes query row t / kInfParts and the operand chunks (four levels
            // each) part, part + kInfParts, ... of it
            const uint32_t row = t / kInfParts, part = t % kInfParts, q = tile * kCacheTile + row;
            float3 p = f3(0.f);
            if (q < n) { const float4 p4 = pos[q]; p = f3(p4.x, p4.y, p4.z); }
#pragma unroll
            for (uint32_t ch = part; ch < 4; ch += kInfParts) {
                __half2 f[4];
                if (q < n) {
                    cache_encode4(c, p, 4u * ch, f);
                } else {
#pragma unroll
                    for (uint32_t j = 0; j < 4; ++j) f[j] = __floats2half2_rn(0.f, 0.f);
                }
                store_chunk(smem + kInfSmemX, row, ch, kCacheIn, f);
            }
        }
        const uint32_t q = tile * kCacheTile + t;  // MLP row of warps 0..3
        // layer 1: D[0:64) = X W1^T
        block_sync_tc();
        if (t == 0 && ok && !c.wait_test) {
            umma_gemm(tmem, s_x, s_w1, kCacheIn, kCacheHidden, false);
            umma_commit(&bar);
        }
        done(true);
        tc_fence_after_sync();
        if (mlp && ok) tmem_relu_to_tile(tlane, 0, smem + kInfSmemH, t);
        // layer 2: D[64:128) = H1 W2^T
        block_sync_tc();
        if (t == 0 && ok) {
            umma_gemm(tmem + 64u, s_h, s_w2, kCacheHidden, kCacheHidden, false);
            umma_commit(&bar);
        }
        done(true);
        tc_fence_after_sync();
        if (mlp && ok) tmem_relu_to_tile(tlane, 64u, smem + kInfSmemH, t);
        // layer 3: D[0:16) = H2 W3^T
        block_sync_tc();
        if (t == 0 && ok) {
            umma_gemm(tmem, s_h, s_w3, kCacheHidden, kCacheOutPad, false);
            umma_commit(&bar);
        }
        done(true);
        tc_fence_after_sync();
        if (mlp && ok) {
            float v[16];
            tmem_ld16(tlane, v);
            if (q < n) {
                if (tput) {
                    const float4 tp = tput[q];
                    const uint32_t slot = __float_as_uint(pos[q].w);
                    const float r = fmaxf(v[0], 0.f) * tp.x, g = fmaxf(v[1], 0.f) * tp.y, b = fmaxf(v[2], 0.f) * tp.z;
                    if (isfinite(r) && isfinite(g) && isfinite(b)) {
                        if (total_fx) {
                            unsigned long long* tf = total_fx + 4 * (size_t)slot;
                            if (r > 0.f) atomicAdd(tf + 0, (unsigned long long)__float2ull_rn(r * S2_FX_SCALE));
                            if (g > 0.f) atomicAdd(tf + 1, (unsigned long long)__float2ull_rn(g * S2_FX_SCALE));
                            if (b > 0.f) atomicAdd(tf + 2, (unsigned long long)__float2ull_rn(b * S2_FX_SCALE));
                        } else {
                            float4 a = accum[slot];
                            a.x += r; a.y += g; a.z += b;
                            accum[slot] = a;
                        }
                    }
                } else {
                    out[q] = make_float4(v[0], v[1], v[2], 0.f);
                }
            }
        }
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        ok = __syncthreads_and(ok);
    }
    if (!ok) {
        // a wait timed out: record it, give an MMA still in flight a bounded time to land, and
        // release TMEM only then
        if (t == 0) atomicOr(c.status, 4);
        if (mlp) mbar_wait(&bar, phase, wait_limit);
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

// ---------------------------------------------------------------- training
// Shared-memory plan of the training kernel (bytes).  The dW GEMMs use M = 128 with the 64 real
// rows of dH2T / dH1T first; rows 64..127 of those A operands read the next 16 KB of the plan (dH1T
// and H2), so the unused accumulator rows hold garbage and every descriptor stays inside the plan.
constexpr uint32_t kTrW = 0;
constexpr uint32_t kTrX = kTrW + kWImageTrainBytes;   // 128 x 32, K-major
constexpr uint32_t kTrXT = kTrX + 8192;              // 32 x 128 (x transposed), B of dW1
constexpr uint32_t kTrH1 = kTrXT + 8192;             // 128 x 64
constexpr uint32_t kTrH1T = kTrH1 + 16384;           // 64 x 128, B of dW2
constexpr uint32_t kTrDH2 = kTrH1T + 16384;          // 128 x 64, A of dH1
constexpr uint32_t kTrDH1 = kTrDH2 + 16384;          // 128 x 64, A of dX
constexpr uint32_t kTrDH2T = kTrDH1 + 16384;         // 64 x 128, A of dW2
constexpr uint32_t kTrDH1T = kTrDH2T + 16384;        // 64 x 128, A of dW1
constexpr uint32_t kTrH2 = kTrDH1T + 16384;          // 128 x 64
constexpr uint32_t kTrDY = kTrH2 + 16384;            // 128 x 3 f32
constexpr uint32_t kTrW3F = kTrDY + 128 * 3 * 4;     // 3 x 64 f32 (f16-rounded W3)
constexpr uint32_t kTrSmemBytes = kTrW3F + 3 * 64 * 4;
// TMEM columns of the training kernel
constexpr uint32_t kTcD1 = 0, kTcD2 = 64, kTcD3 = 128, kTcDH1 = 192, kTcDX = 256, kTcDW2 = 320, kTcDW1 = 384;
constexpr uint32_t kTrTmemCols = 512;

S2D void st_half(uint8_t* base, uint32_t off, float v) { *(__half*)(base + off) = __float2half_rn(v); }
S2D float ld_half(const uint8_t* base, uint32_t off) { return __half2float(*(const __half*)(base + off)); }

// Bounded wait + state bookkeeping shared by the training steps.
struct TcSync {
    uint64_t* bar;
    uint32_t phase;
    bool ok;
    // wait for the committed MMAs; `ok` is made warp-uniform so the collective tcgen05.ld calls
    // that it guards are executed by whole warps
    S2D void mma_done() {
        const bool w = ok && mbar_wait(bar, phase);
        if (w) phase ^= 1u;
        ok = __all_sync(0xffffffffu, w);
        tc_fence_after_sync();
    }
};


// One pass over n training records (position, target radiance): forward, relative L2 loss
// sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) / 3 per record (denominator not differentiated), backward
// through the MLP on the tensor cores, and the summed per-record gradients of the weights
// (grad_w) and of the table entries (grad_t, scattered with atomics).  128 threads,
// kTrSmemBytes dynamic shared memory, 512 TMEM columns (one CTA per SM).
__global__ void __launch_bounds__(128, 1) k_cache_train(const __grid_constant__ CacheDev c, const float4* __restrict__ pos,
                                                        const float4* __restrict__ target, uint32_t n,
                                                        const uint32_t* __restrict__ n_dev) {
    if (n_dev) n = min(n, *n_dev);
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ float loss_part[4];
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
    for (uint32_t i = t; i < kWImageTrainBytes / 16; i += 128) ((uint4*)(smem + kTrW))[i] = c.wimage[i];
    if (warp == 0) {
        tmem_alloc(&tmem_base, kTrTmemCols);
        tmem_relinquish();
    }
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    block_sync_tc();
    float* dy_s = (float*)(smem + kTrDY);
    float* w3f = (float*)(smem + kTrW3F);
    for (uint32_t e = t; e < kCacheW3; e += 128) {
        const uint32_t ch = e / kCacheHidden, i = e % kCacheHidden;
        w3f[e] = ld_half(smem, kTrW + kW1Bytes + kW2Bytes + kmaj_offset(ch, i, kCacheHidden));
    }
    const uint32_t tmem = tmem_base;
    const uint32_t tlane = tmem + ((32u * (warp & 3u)) << 16);
    const uint32_t s0 = smem_addr(smem);
    const uint32_t s_w1 = s0 + kTrW, s_w2 = s_w1 + kW1Bytes, s_w3 = s_w2 + kW2Bytes, s_w2t = s_w3 + kW3Bytes,
                   s_w1t = s_w2t + kW2TBytes;
    TcSync sy{&bar, 0u, true};
    float acc3[2] = {0.f, 0.f};  // dW3 entries t and t + 128 (CUDA cores)
    float loss = 0.f;
    bool first = true;
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    for (uint32_t tile = blockIdx.x; tile < tiles && sy.ok; tile += gridDim.x) {
        const uint32_t q = tile * kCacheTile + t;
        const bool valid = q < n;
        float3 p = f3(0.f), tg = f3(0.f);
        if (valid) {
            const float4 a = pos[q], b = target[q];
            p = f3(a.x, a.y, a.z);
            tg = f3(b.x, b.y, b.z);
        }
        // ---- forward
        __half2 f[kCacheLevels];
        if (valid) cache_encode(c, p, f);
        else
#pragma unroll
            for (uint32_t l = 0; l < kCacheLevels; ++l) f[l] = __floats2half2_rn(0.f, 0.f);
#pragma unroll
        for (uint32_t ch = 0; ch < 4; ++ch) store_chunk(smem + kTrX, t, ch, kCacheIn, f + 4 * ch);
#pragma unroll
        for (uint32_t l = 0; l < kCacheLevels; ++l) {
            *(__half*)(smem + kTrXT + kmaj_offset(2 * l, t, 128)) = __low2half(f[l]);
            *(__half*)(smem + kTrXT + kmaj_offset(2 * l + 1, t, 128)) = __high2half(f[l]);
        }
        block_sync_tc();
        if (t == 0) {
            umma_gemm(tmem + kTcD1, s0 + kTrX, s_w1, kCacheIn, kCacheHidden, false);
            umma_commit(&bar);
        }
        sy.mma_done();
        if (sy.ok) {
#pragma unroll
            for (uint32_t g = 0; g < 4; ++g) {
                float v[16];
                tmem_ld16(tlane + kTcD1 + 16u * g, v);
                __half2 h[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) h[i] = __floats2half2_rn(fmaxf(v[2 * i], 0.f), fmaxf(v[2 * i + 1], 0.f));
                store_chunk(smem + kTrH1, t, 2 * g, kCacheHidden, h);
                store_chunk(smem + kTrH1, t, 2 * g + 1, kCacheHidden, h + 4);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    *(__half*)(smem + kTrH1T + kmaj_offset(16 * g + 2 * i, t, 128)) = __low2half(h[i]);
                    *(__half*)(smem + kTrH1T + kmaj_offset(16 * g + 2 * i + 1, t, 128)) = __high2half(h[i]);
                }
            }
        }
        block_sync_tc();
        if (t == 0 && sy.ok) {
            umma_gemm(tmem + kTcD2, s0 + kTrH1, s_w2, kCacheHidden, kCacheHidden, false);
            umma_commit(&bar);
        }
        sy.mma_done();
        if (sy.ok) tmem_relu_to_tile(tlane, kTcD2, smem + kTrH2, t);
        block_sync_tc();
        if (t == 0 && sy.ok) {
            umma_gemm(tmem + kTcD3, s0 + kTrH2, s_w3, kCacheHidden, kCacheOutPad, false);
            umma_commit(&bar);
        }
        sy.mma_done();
        // ---- loss and output gradient; dH2 = (dY W3) masked by h2 > 0
        float dy[3] = {0.f, 0.f, 0.f};
        if (sy.ok) {
            float v[16];
            tmem_ld16(tlane + kTcD3, v);
            if (valid) {
                const float yt[3] = {tg.x, tg.y, tg.z};
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float d = v[ch] - yt[ch], den = v[ch] * v[ch] + 0.01f;
                    loss += d * d / den / 3.f;
                    dy[ch] = fminf(fmaxf(2.f * d / den / 3.f, -1e4f), 1e4f);
                }
            }
        }
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) dy_s[3 * t + ch] = dy[ch];
#pragma unroll
        for (uint32_t g = 0; g < 8; ++g) {
            const uint4 hv = *(const uint4*)(smem + kTrH2 + kmaj_offset(t, 8 * g, kCacheHidden));
            const __half* hh = (const __half*)&hv;
            __half2 o[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float r2[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const uint32_t i = 8 * g + 2 * j + u;
                    const float s = dy[0] * w3f[i] + dy[1] * w3f[64 + i] + dy[2] * w3f[128 + i];
                    r2[u] = __half2float(hh[2 * j + u]) > 0.f ? s * kCacheGradScale : 0.f;
                }
                o[j] = __floats2half2_rn(r2[0], r2[1]);
                *(__half*)(smem + kTrDH2T + kmaj_offset(8 * g + 2 * j, t, 128)) = __low2half(o[j]);
                *(__half*)(smem + kTrDH2T + kmaj_offset(8 * g + 2 * j + 1, t, 128)) = __high2half(o[j]);
            }
            store_chunk(smem + kTrDH2, t, g, kCacheHidden, o);
        }
        block_sync_tc();
        // dW3 on the CUDA cores: entry e = (channel e / 64, input e % 64), summed over the tile
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t e = t + 128u * k;
            if (e < kCacheW3) {
                const uint32_t ch = e / kCacheHidden, i = e % kCacheHidden;
                float a = 0.f;
                for (uint32_t b = 0; b < kCacheTile; ++b) a += dy_s[3 * b + ch] * ld_half(smem + kTrH2, kmaj_offset(b, i, kCacheHidden));
                acc3[k] += a;
            }
        }
        if (t == 0 && sy.ok) {
            umma_gemm(tmem + kTcDH1, s0 + kTrDH2, s_w2t, kCacheHidden, kCacheHidden, false);
            umma_gemm(tmem + kTcDW2, s0 + kTrDH2T, s0 + kTrH1T, kCacheTile, kCacheHidden, !first);
            umma_commit(&bar);
        }
        sy.mma_done();
        // dH1 = (dH2 W2) masked by h1 > 0
        if (sy.ok) {
#pragma unroll
            for (uint32_t g = 0; g < 4; ++g) {
                float v[16];
                tmem_ld16(tlane + kTcDH1 + 16u * g, v);
                const uint4 m0 = *(const uint4*)(smem + kTrH1 + kmaj_offset(t, 16 * g, kCacheHidden));
                const uint4 m1 = *(const uint4*)(smem + kTrH1 + kmaj_offset(t, 16 * g + 8, kCacheHidden));
                const __half* h0 = (const __half*)&m0;
                const __half* h1 = (const __half*)&m1;
                __half2 o[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float a = __half2float((2 * i < 8) ? h0[2 * i] : h1[2 * i - 8]) > 0.f ? v[2 * i] : 0.f;
                    const float b = __half2float((2 * i + 1 < 8) ? h0[2 * i + 1] : h1[2 * i + 1 - 8]) > 0.f ? v[2 * i + 1] : 0.f;
                    o[i] = __floats2half2_rn(a, b);
                    *(__half*)(smem + kTrDH1T + kmaj_offset(16 * g + 2 * i, t, 128)) = __low2half(o[i]);
                    *(__half*)(smem + kTrDH1T + kmaj_offset(16 * g + 2 * i + 1, t, 128)) = __high2half(o[i]);
                }
                store_chunk(smem + kTrDH1, t, 2 * g, kCacheHidden, o);
                store_chunk(smem + kTrDH1, t, 2 * g + 1, kCacheHidden, o + 4);
            }
        }
        block_sync_tc();
        if (t == 0 && sy.ok) {
            umma_gemm(tmem + kTcDX, s0 + kTrDH1, s_w1t, kCacheHidden, kCacheIn, false);
            umma_gemm(tmem + kTcDW1, s0 + kTrDH1T, s0 + kTrXT, kCacheTile, kCacheIn, !first);
            umma_commit(&bar);
        }
        sy.mma_done();
        // dX -> table gradients (same corners and weights as the encoding)
        float dx[32];
        if (sy.ok) {
            tmem_ld16(tlane + kTcDX, dx);
            tmem_ld16(tlane + kTcDX + 16u, dx + 16);
        }
        if (sy.ok && valid) {
            const float3 u = cache_unit(c, p);
            for (uint32_t l = 0; l < kCacheLevels; ++l) {
                const float r = c.res[l];
                const float fx = u.x * r, fy = u.y * r, fz = u.z * r;
                const float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
                const float wx = fx - ix, wy = fy - iy, wz = fz - iz;
                const uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
                const float g0 = dx[2 * l] / kCacheGradScale, g1 = dx[2 * l + 1] / kCacheGradScale;
                float* gt = c.grad_t + ((size_t)l << c.log2_table) * 2;
                for (uint32_t k = 0; k < 8; ++k) {
                    const uint32_t ddx = k & 1u, ddy = (k >> 1) & 1u, ddz = k >> 2;
                    const float w = (ddx ? wx : 1.f - wx) * (ddy ? wy : 1.f - wy) * (ddz ? wz : 1.f - wz);
                    const uint32_t idx = cache_index(c, l, x0 + ddx, y0 + ddy, z0 + ddz);
                    atomicAdd(gt + 2 * idx, w * g0);
                    atomicAdd(gt + 2 * idx + 1, w * g1);
                }
            }
        }
        first = false;
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        sy.ok = __syncthreads_and(sy.ok);
    }
    // ---- weight gradients leave TMEM (rows 0..63 = output features live in warps 0 and 1)
    if (sy.ok && !first && warp < 2) {
        for (uint32_t g = 0; g < 4; ++g) {
            float v[16];
            tmem_ld16(tlane + kTcDW2 + 16u * g, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) atomicAdd(c.grad_w + kCacheW1 + t * kCacheHidden + 16 * g + i, v[i] / kCacheGradScale);
        }
        for (uint32_t g = 0; g < 2; ++g) {
            float v[16];
            tmem_ld16(tlane + kTcDW1 + 16u * g, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) atomicAdd(c.grad_w + t * kCacheIn + 16 * g + i, v[i] / kCacheGradScale);
        }
    }
    if (sy.ok && !first) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t e = t + 128u * k;
            if (e < kCacheW3) atomicAdd(c.grad_w + kCacheW1 + kCacheW2 + e, acc3[k]);
        }
    }
    // loss: warp sums, then one atomic per CTA
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) loss_part[warp] = loss;
    __syncthreads();
    if (t == 0) atomicAdd(c.loss_sum, loss_part[0] + loss_part[1] + loss_part[2] + loss_part[3]);
    if (!sy.ok) {
        if (t == 0) atomicOr(c.status, 4);
        mbar_wait(&bar, sy.phase);
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kTrTmemCols);
}

// Adam on the f32 master parameters with the summed gradients scaled by 1/n; clears the gradients.
// n_dev (optional): the record count is read on the device (capped at n_cap) instead of inv_n.
__global__ void k_cache_adam(float* __restrict__ param, float* __restrict__ grad, float* __restrict__ m,
                             float* __restrict__ v, size_t count, float inv_n, const uint32_t* __restrict__ n_dev,
                             uint32_t n_cap, float lr, float b1, float b2, float eps, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (n_dev) inv_n = 1.f / (float)max(1u, min(*n_dev, n_cap));
    const float g = grad[i] * inv_n;
    grad[i] = 0.f;
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    param[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Lazy Adam on the table (TensorFlow's LazyAdam semantics): an entry whose summed gradient is zero
// this step (no record touched it) keeps its parameters and moments; touched entries take the Adam
// step on their f32 masters, clear their gradient and refresh their f16 copy in the same pass, so
// untouched entries cost an 8-byte gradient read.  One thread per entry (two features).
__global__ void k_cache_adam_table(float2* __restrict__ param, float2* __restrict__ grad, float2* __restrict__ m,
                                   float2* __restrict__ v, __half2* __restrict__ t16, uint32_t entries, float inv_n,
                                   const uint32_t* __restrict__ n_dev, uint32_t n_cap, float lr, float b1, float b2,
                                   float eps, float c1, float c2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= entries) return;
    const float2 g0 = grad[i];
    if (g0.x == 0.f && g0.y == 0.f) return;
    if (n_dev) inv_n = 1.f / (float)max(1u, min(*n_dev, n_cap));
    grad[i] = make_float2(0.f, 0.f);
    const float gx = g0.x * inv_n, gy = g0.y * inv_n;
    float2 mi = m[i], vi = v[i], pi = param[i];
    mi.x = b1 * mi.x + (1.f - b1) * gx;
    mi.y = b1 * mi.y + (1.f - b1) * gy;
    vi.x = b2 * vi.x + (1.f - b2) * gx * gx;
    vi.y = b2 * vi.y + (1.f - b2) * gy * gy;
    pi.x -= lr * (mi.x / c1) / (sqrtf(vi.x / c2) + eps);
    pi.y -= lr * (mi.y / c1) / (sqrtf(vi.y / c2) + eps);
    m[i] = mi;
    v[i] = vi;
    param[i] = pi;
    t16[i] = __floats2half2_rn(pi.x, pi.y);
}

}  // namespace s2
