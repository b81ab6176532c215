// Internal context of the C ABI: one device, one stream, device-resident scene and BVH.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/stratum2.h"
#include "s2_bvh_build.h"
#include "s2_scene.cuh"

namespace s2 {

// A device allocation owned by the context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct RenderState;  // wavefront queues and accumulators (s2_render.cu)
struct CacheState;   // learned radiance cache parameters and optimiser state (s2_cache.cu)
struct PostState;    // temporal-accumulation history and tonemap scratch (s2_post.cu)
struct VcmState;     // the VCM renderer's direct-illumination reservoir grids (s2_vcm.cu)

struct HostImage {
    uint32_t w = 0, h = 0;
    std::vector<float> rgba;  // 4 floats per texel
};

}  // namespace s2

struct S2Context {
    int device = 0;
    cudaStream_t stream = nullptr;       // the stream work is issued on
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string last_error;
    std::vector<s2::DevBuf> scene_bufs;  // freed on re-upload / destroy
    std::vector<s2::DevBuf> bvh_bufs;
    bool has_scene = false, has_bvh = false;
    uint64_t bvh_node_count = 0;           // 128-byte BVH8 nodes in bvh_bufs

    // host copies needed by the BVH build
    std::vector<float> tri_v0, tri_v1, tri_v2;
    std::vector<uint32_t> tri_inst, tri_prim;
    std::vector<uint32_t> inst_tri_offset;  // flattened triangle base per instance
    std::vector<uint8_t> inst_alpha;        // 1: the instance's triangles need the alpha test

    // device scene description (pointers into scene_bufs / bvh_bufs)
    DevScene scene{};
    std::vector<DevImage> images_host;      // device-side descriptors, host copy
    std::vector<uint32_t> image_channels;   // channel count of each uploaded image
    DevImage* images_dev = nullptr;
    DevImage env_fp_host{};                 // S2_FLAG_ENV_FOOTPRINT_PDF tables of the environment image
    DevImage* env_fp_dev = nullptr;
    uint8_t** vbufs_dev = nullptr;
    int env_image = -1;

    s2::RenderState* render = nullptr;
    s2::CacheState* cache = nullptr;
    s2::PostState* post = nullptr;
    s2::VcmState* vcm = nullptr;
    S2Tuning tuning{};                      // wavefront renderer tuning (zeros = defaults)
    int* status_dev = nullptr;              // device status word (stack/queue overflow, timeouts)
};

namespace s2 {
int set_error(S2Context* ctx, int code, const std::string& msg);
int check_cuda(S2Context* ctx, cudaError_t e, const char* what);
void* dev_alloc(S2Context* ctx, std::vector<DevBuf>& owner, size_t bytes);
void free_bufs(std::vector<DevBuf>& bufs);
void destroy_render_state(S2Context* ctx);
void destroy_cache_state(S2Context* ctx);
void destroy_post_state(S2Context* ctx);
void destroy_vcm_state(S2Context* ctx);
// baked shading records of the current BVH (s2_render.cu), allocated into `owner`
int bake_shading_records(S2Context* ctx, std::vector<DevBuf>& owner);
// radiance cache entry points used by the renderer (s2_cache.cu)
int cache_apply_device(S2Context* ctx, const float4* pos, const float4* tput, uint32_t cap, const uint32_t* n_dev,
                       float4* accum, unsigned long long* total_fx = nullptr);
void cache_prepare_device(S2Context* ctx);
int cache_backward_device(S2Context* ctx, const float4* pos, const float4* target, uint32_t n, const uint32_t* n_dev);
int cache_adam_device(S2Context* ctx, uint32_t n, const uint32_t* n_dev);
}  // namespace s2
