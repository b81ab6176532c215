// BVH8 layout shared by the host builder and the device traversal.
//
// The reference has no BVH of its own: it builds Vulkan acceleration structures
// (src/App/Scene.cpp:17-55, BLAS :560-589, TLAS :726-754) and traverses them with hardware ray
// queries (src/Shaders/common/intersection.hlsli:74-75).  B200 has no RT cores, so this file
// defines a compressed 8-wide BVH (quantized child boxes in the style of Ylitie, Karras and
// Laine, HPG 2017) over world-space triangles.  All mesh instances are flattened into one BVH:
// with 180 GB of HBM per GPU the memory cost of pre-transformed triangles is irrelevant and the
// traversal never crosses an instance boundary.
#pragma once
#include <stdint.h>

#define S2_BVH_WIDTH 8
#define S2_BVH_MAX_LEAF_TRIS 3
// Traversal stack: entries [0, S2_STACK_SMEM) live in shared memory, the rest in local memory.
// The builder guarantees tree depth <= S2_STACK_DEPTH.
#define S2_STACK_SMEM 16
#define S2_STACK_DEPTH 64

// One node = 80 bytes of payload on its own 128-byte line (so a node fetch touches exactly
// three 32-byte L2 sectors).
//   word 0-2   float origin p of the quantization grid
//   word 3     exponent bytes ex, ey, ez (biased like IEEE float: scale = 2^(e-127)), imask
//   word 4     child_base: index of the first internal child (internal children are contiguous
//              in slot order)
//   word 5     tri_base: index of the first triangle record of this node's leaf slots
//   word 6-7   meta[8]: leaf slot: (count << 5) | offset (count 1..3, offset 0..23);
//              internal slot or empty slot: 0
//   word 8-19  qlo_x[8], qlo_y[8], qlo_z[8], qhi_x[8], qhi_y[8], qhi_z[8]
// Empty slots carry qlo = 255, qhi = 0 on every axis (an empty box).
// Slot s holds the child that is nearest for rays whose direction octant is s (bit i set when
// direction component i is negative), so visiting bit positions (slot ^ ray_octant) in
// increasing order is approximately front to back.
struct alignas(128) S2BvhNode {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlo[3][8];
    uint8_t qhi[3][8];
    uint8_t pad[48];
};
static_assert(sizeof(S2BvhNode) == 128, "node must fill one 128-byte line");

// One triangle record = 48 bytes: world-space vertices, with the instance and primitive index
// in the w components: {v0, instance}, {v1, primitive}, {v2, flattened triangle id}.  Bit 31 of
// the flattened id marks triangles whose material has an alpha mask with texels below its cutoff
// (the reference builds those as non-opaque geometry, Scene.cpp:575, and tests them in the ray
// query, intersection.hlsli:125-146).
struct alignas(16) S2TriRecord {
    float v0[3]; uint32_t instance;
    float v1[3]; uint32_t primitive;
    float v2[3]; uint32_t flat_id;
};
static_assert(sizeof(S2TriRecord) == 48, "triangle record is 48 bytes");
#define S2_TRI_ALPHA_TESTED 0x80000000u
