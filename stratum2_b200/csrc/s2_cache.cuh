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

struct CacheDev {
    const __half2* table;        // [levels][2^log2_table] feature pairs
    uint32_t log2_table;
    float res[kCacheLevels];     // grid resolution per level
    uint32_t dense[kCacheLevels];// 1: level indexed densely ((res+1)^3 <= table size)
    float3 box_min, box_inv_extent;
    const uint4* wimage;         // kWImageBytes, the three weight tiles in operand layout
    int* status;                 // bit 2: a tensor-core wait timed out
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

S2D uint32_t cache_index(const CacheDev& c, uint32_t level, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t mask = (1u << c.log2_table) - 1u;
    if (c.dense[level]) {
        const uint32_t n = (uint32_t)c.res[level] + 1u;
        return (x + n * (y + n * z)) & mask;
    }
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & mask;
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

// Shared-memory plan of the inference kernel (bytes): weights, input tile, hidden tile.
constexpr uint32_t kInfSmemW = 0;
constexpr uint32_t kInfSmemX = kWImageBytes;                         // 128 x 32 f16
constexpr uint32_t kInfSmemH = kInfSmemX + kCacheTile * kCacheIn * 2; // 128 x 64 f16
constexpr uint32_t kInfSmemBytes = kInfSmemH + kCacheTile * kCacheHidden * 2;

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

// Radiance cache inference: out[i] = MLP(encode(pos[i])), raw (unclamped) outputs.
// Persistent: grid-stride over tiles of 128 queries; 128 threads; kInfSmemBytes dynamic smem.
__global__ void __launch_bounds__(128, 1) k_cache_infer(const __grid_constant__ CacheDev c, const float4* __restrict__ pos,
                                                        uint32_t n, float4* __restrict__ out) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    const uint32_t t = threadIdx.x, warp = t >> 5;
    // stage the weight images
    for (uint32_t i = t; i < kWImageBytes / 16; i += 128) ((uint4*)(smem + kInfSmemW))[i] = c.wimage[i];
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
    const uint32_t tiles = (n + kCacheTile - 1) / kCacheTile;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t q = tile * kCacheTile + t;
        __half2 f[kCacheLevels];
        if (q < n) {
            const float4 p = pos[q];
            cache_encode(c, f3(p.x, p.y, p.z), f);
        } else {
#pragma unroll
            for (uint32_t l = 0; l < kCacheLevels; ++l) f[l] = __floats2half2_rn(0.f, 0.f);
        }
#pragma unroll
        for (uint32_t ch = 0; ch < 4; ++ch) store_chunk(smem + kInfSmemX, t, ch, kCacheIn, f + 4 * ch);
        // layer 1: D[0:64) = X W1^T
        fence_smem_async();
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        if (t == 0) {
            umma_gemm(tmem, s_x, s_w1, kCacheIn, kCacheHidden, false);
            umma_commit(&bar);
        }
        ok = mbar_wait(&bar, phase);
        if (ok) phase ^= 1u;
        tc_fence_after_sync();
        if (ok) tmem_relu_to_tile(tlane, 0, smem + kInfSmemH, t);
        // layer 2: D[64:128) = H1 W2^T
        fence_smem_async();
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        if (t == 0 && ok) {
            umma_gemm(tmem + 64u, s_h, s_w2, kCacheHidden, kCacheHidden, false);
            umma_commit(&bar);
        }
        ok = ok && mbar_wait(&bar, phase);
        if (ok) phase ^= 1u;
        tc_fence_after_sync();
        if (ok) tmem_relu_to_tile(tlane, 64u, smem + kInfSmemH, t);
        // layer 3: D[0:16) = H2 W3^T
        fence_smem_async();
        tc_fence_before_sync();
        __syncthreads();
        tc_fence_after_sync();
        if (t == 0 && ok) {
            umma_gemm(tmem, s_h, s_w3, kCacheHidden, kCacheOutPad, false);
            umma_commit(&bar);
        }
        ok = ok && mbar_wait(&bar, phase);
        if (ok) phase ^= 1u;
        tc_fence_after_sync();
        if (ok) {
            float v[16];
            tmem_ld16(tlane, v);
            if (q < n) out[q] = make_float4(v[0], v[1], v[2], 0.f);
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
        mbar_wait(&bar, phase);
    }
    tc_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

}  // namespace s2
