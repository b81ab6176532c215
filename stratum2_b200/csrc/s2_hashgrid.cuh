// World-space hash grid of ReSTIR DI reservoirs (src/Shaders/common/hashgrid.hlsli:14-119,
// src/App/GpuHashGrid.cpp:17-111): cells keyed by the pcg hash of the quantized position with an
// xxhash32 checksum and 32-step linear probing; items are appended with atomics, then a prefix sum
// over the per-cell counters and a sort by (cell, record content) list them by cell.  The renderer keeps two grids:
// the previous frame's (read) and the current frame's (appended to, built at the end of the call).
#pragma once
#include "s2_math.cuh"

// HashGridData (testrenderer.slang:152-168) without the light-vertex-cache part: the vertex (as
// an object-space position on a triangle), its reservoir and its local incident direction.
struct ReservoirRecord {
    float3 local_pos;
    uint32_t instance;
    float4 rnd;            // the light sample (the 4 random numbers that define it)
    float target_pdf;      // cached target pdf of the sample at this vertex
    float W;               // integration (contribution) weight
    float M;               // sample count (capped)
    uint32_t primitive;
    float3 local_dir_in;
    float pad;
};

struct HashGridDev {
    uint32_t* checksums;
    uint32_t* cell_counters;
    uint32_t* other;            // [0] appended items, [1] prefix-sum counter
    uint2* append_indices;      // (cell, index in cell) in append order
    ReservoirRecord* data;
    uint32_t* indices;          // per-cell offset into data_indices
    uint32_t* data_indices;
    uint32_t cell_count;
    uint32_t max_size;
    float min_cell_size;
    float cell_pixel_radius;
    float3 camera_position;
    float distance_scale;
};

// GetCellSize (hashgrid.hlsli:43-49)
S2D float hg_cell_size(const HashGridDev& g, float3 pos) {
    if (g.cell_pixel_radius <= 0.f) return g.min_cell_size;
    const float step = length(g.camera_position - pos) * g.distance_scale;
    // uint(log2(x)) of a negative value (x < 1) is taken as 0, the GPUs' saturating conversion
    const float l = log2f(step / g.min_cell_size);
    const uint32_t e = l > 0.f ? min((uint32_t)l, 31u) : 0u;
    return g.min_cell_size * (float)(1u << e);
}

// FindCellIndex (hashgrid.hlsli:51-75); returns 0xffffffff when not found / full.
template <bool INSERT>
S2D uint32_t hg_find_cell(const HashGridDev& g, float3 pos, float cell_size) {
    const int px = (int)floorf(pos.x / cell_size), py = (int)floorf(pos.y / cell_size), pz = (int)floorf(pos.z / cell_size);
    const uint32_t cs = __float_as_uint(cell_size);
    const uint32_t checksum = max(1u, xxhash32(xxhash32(cs) + xxhash32((uint32_t)pz + xxhash32((uint32_t)py + xxhash32((uint32_t)px)))));
    const uint32_t base = (pcg_hash(pcg_hash(cs) + pcg_hash((uint32_t)pz + pcg_hash((uint32_t)py + pcg_hash((uint32_t)px))))) % g.cell_count;
    for (uint32_t i = 0; i < 32; ++i) {
        const uint32_t cell = (base + i) % g.cell_count;
        if (INSERT) {
            const uint32_t prev = atomicCAS(&g.checksums[cell], 0u, checksum);
            if (prev == 0u || prev == checksum) return cell;
        } else {
            if (g.checksums[cell] == checksum) return cell;
        }
    }
    return 0xffffffffu;
}

// Append (hashgrid.hlsli:77-97): returns the record's data index, 0xffffffff when the grid is full
// (grids with a wider payload store it in their own array at that index).
S2D uint32_t hg_append(const HashGridDev& g, float3 pos, const ReservoirRecord& rec) {
    const uint32_t cell = hg_find_cell<true>(g, pos, hg_cell_size(g, pos));
    if (cell == 0xffffffffu) return 0xffffffffu;
    const uint32_t idx = atomicAdd(&g.other[0], 1u);
    if (idx >= g.max_size) return 0xffffffffu;
    const uint32_t in_cell = atomicAdd(&g.cell_counters[cell], 1u);
    g.append_indices[idx] = make_uint2(cell, in_cell);
    g.data[idx] = rec;
    return idx;
}

// Building the grid (the work of ComputeIndices and Swizzle, hashgrid.hlsli:101-119), so that the
// order of the records inside a cell does not depend on the order of the atomic appends:
//  * k_hg_scan: each cell's offset is the exclusive prefix sum of the cell counters in cell order
//    (one block: per-thread runs of cells, then a block scan of the run totals), where the
//    reference adds them with an atomic counter in arrival order;
//  * k_hg_keys: a 64-bit key per appended record, its cell above a hash of its content, and
//    unused slots in a cell past the last;
//  * a radix sort of (key, record index) pairs (cub::DeviceRadixSort, in s2_render.cu) lists the
//    records by cell, and inside a cell by content: data_indices[indices[c] + k] is the k-th
//    record of cell c in an order fixed by the records themselves.
constexpr uint32_t kHgScanThreads = 1024;
__global__ void __launch_bounds__(kHgScanThreads) k_hg_scan(HashGridDev g) {
    __shared__ uint32_t part[kHgScanThreads];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (g.cell_count + kHgScanThreads - 1) / kHgScanThreads;
    const uint32_t c0 = t * per, c1 = min(c0 + per, g.cell_count);
    uint32_t sum = 0;
    for (uint32_t c = c0; c < c1; ++c) sum += g.cell_counters[c];
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < kHgScanThreads; off <<= 1) {  // inclusive Hillis-Steele scan
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t c = c0; c < c1; ++c) {
        g.indices[c] = run;
        run += g.cell_counters[c];
    }
}

S2D uint32_t hg_record_hash(const ReservoirRecord& r) {
    uint32_t h = xxhash32(r.instance ^ 0x9e3779b9u);
    h = xxhash32(h ^ r.primitive);
    h = xxhash32(h ^ __float_as_uint(r.local_pos.x));
    h = xxhash32(h ^ __float_as_uint(r.local_pos.y));
    h = xxhash32(h ^ __float_as_uint(r.local_pos.z));
    h = xxhash32(h ^ __float_as_uint(r.rnd.x));
    h = xxhash32(h ^ __float_as_uint(r.rnd.y));
    h = xxhash32(h ^ __float_as_uint(r.rnd.z));
    h = xxhash32(h ^ __float_as_uint(r.rnd.w));
    return xxhash32(h ^ __float_as_uint(r.W));
}

__global__ void k_hg_keys(HashGridDev g, unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.max_size) return;
    const uint32_t n = min(g.other[0], g.max_size);
    vals[i] = i;
    keys[i] = i < n ? (((unsigned long long)g.append_indices[i].x << 32) | hg_record_hash(g.data[i]))
                    : (((unsigned long long)g.cell_count << 32) | 0xffffffffull);
}
