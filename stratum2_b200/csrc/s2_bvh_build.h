// Host BVH8 builder interface.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "s2_bvh.h"

namespace s2 {

struct BuildInput {
    uint32_t count = 0;            // triangles
    const float* v0 = nullptr;     // 3*count world-space vertex positions
    const float* v1 = nullptr;
    const float* v2 = nullptr;
    const uint32_t* instance = nullptr;
    const uint32_t* primitive = nullptr;
};

struct BuildParams {
    uint32_t max_leaf_size = 3;
    uint32_t sah_bins = 32;
    uint32_t threads = 0;
    uint32_t collapse = 0;  // S2_BVH_COLLAPSE_SAH (0): cost-optimal collapse; S2_BVH_COLLAPSE_GREEDY (1)
};

struct BuildOutput {
    std::vector<S2BvhNode> nodes;
    std::vector<S2TriRecord> tris;
    uint32_t max_depth = 0;
    uint64_t leaf_slots = 0;
    double sah_cost = 0;
    double seconds = 0;
};

// Returns 0 on success, -1 with `err` set otherwise.
int build_bvh8(const BuildInput& in, const BuildParams& prm, BuildOutput& out, std::string& err);

}  // namespace s2
