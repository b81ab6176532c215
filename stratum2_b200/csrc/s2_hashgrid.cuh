// World-space hash grid of ReSTIR DI reservoirs (src/Shaders/common/hashgrid.hlsli:14-119,
// src/App/GpuHashGrid.cpp:17-111): cells keyed by the pcg hash of the quantized position with an
// xxhash32 checksum and 32-step linear probing; items are appended with atomics, then a prefix sum
// over the per-cell counters and a swizzle sort them by cell.  The renderer keeps two grids:
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

// Append (hashgrid.hlsli:77-97)
S2D void hg_append(const HashGridDev& g, float3 pos, const ReservoirRecord& rec) {
    const uint32_t cell = hg_find_cell<true>(g, pos, hg_cell_size(g, pos));
    if (cell == 0xffffffffu) return;
    const uint32_t idx = atomicAdd(&g.other[0], 1u);
    if (idx >= g.max_size) return;
    const uint32_t in_cell = atomicAdd(&g.cell_counters[cell], 1u);
    g.append_indices[idx] = make_uint2(cell, in_cell);
    g.data[idx] = rec;
}

// ComputeIndices (hashgrid.hlsli:101-108): one thread per cell
__global__ void k_hg_compute_indices(HashGridDev g) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.cell_count) return;
    g.indices[c] = atomicAdd(&g.other[1], g.cell_counters[c]);
}

// Swizzle (hashgrid.hlsli:111-119): one thread per appended item
__global__ void k_hg_swizzle(HashGridDev g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = min(g.other[0], g.max_size);
    if (i >= n) return;
    const uint2 a = g.append_indices[i];
    g.data_indices[g.indices[a.x] + a.y] = i;
}
