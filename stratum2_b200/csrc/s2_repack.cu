// s2_repack_metallic_roughness: the texture repack of a glTF metallic-roughness material on the
// device, as the reference's from_gltf_pbr compute pass does it (src/Shaders/kernels/
// convert_material.slang:33-69, dispatched by makeMetallicRoughnessMaterial, src/App/Scene.cpp:
// 195-208): per texel, the PackedMaterialData of the base colour, metallic-roughness and emission
// textures, stored as the four packed words' RGBA8 images (PackedMaterialData::Store,
// src/Shaders/common/material.hlsli:113-118), the base colour's alpha as the alpha-mask image and
// the smallest alpha below 1 as an 8-bit value.
//
// Inputs are the decoded 8-bit texels (RGBA8, the loader expands grey and RGB).  The reference
// samples the base colour and emission through sRGB texture formats, so the hardware decodes them
// to linear before the setters quantise them again; here the decode is srgbToRgb
// (compat/common.h:81-86) evaluated in f64 into a 256-entry shared-memory table, and the
// quantisation (material_data.h:51-73: floor(saturate(v) * 255 + 0.5)) and the emission's
// normalisation by its largest channel (setEmission) are done in f64 as well, so the result is the
// exact value of those formulas for every 8-bit input.
//
// One thread per texel over a grid-stride loop; the kernel reads 4 bytes per present texture and
// writes 4 x 16 bytes of packed images plus 4 bytes of alpha per texel: HBM-bound byte work.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "s2_context.h"

using s2::check_cuda;
using s2::set_error;

namespace {

constexpr uint32_t kRepackBlock = 256;

struct RepackArgs {
    uint32_t n;
    const uchar4* base;   // sRGB base colour + linear alpha, or null (1)
    const uchar4* mr;     // linear metallic (b) / roughness (g), or null (1)
    const uchar4* em;     // sRGB emission, or null (1)
    float4* out0;         // base colour, specular
    float4* out1;         // emission / max, sheen
    float4* out2;         // metallic, roughness, anisotropic, subsurface
    float4* out3;         // clearcoat, clearcoat gloss, transmission, eta
    float* alpha;         // base colour alpha (null: not written)
    uint32_t* min_alpha;  // min over texels with alpha < 1 of the 8-bit alpha
};

// setX's quantisation followed by D3DX_R8G8B8A8_UNORM_to_FLOAT4's byte / 255 (IEEE division)
__device__ __forceinline__ float unorm8(double v) {
    v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
    return __fdiv_rn((float)floor(v * 255.0 + 0.5), 255.f);
}

__global__ void __launch_bounds__(kRepackBlock) k_repack_gltf_pbr(const RepackArgs A) {
    __shared__ double lin[256];
    for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
        const double c = i / 255.0;
        lin[i] = c <= 0.04045 ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4);
    }
    __syncthreads();
    const float one = 1.f;  // unorm8(1)
    uint32_t amin = 255u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < A.n; t += stride) {
        const uchar4 d = A.base ? A.base[t] : make_uchar4(255, 255, 255, 255);
        A.out0[t] = make_float4(unorm8(lin[d.x]), unorm8(lin[d.y]), unorm8(lin[d.z]), one);
        if (A.base) {
            if (A.alpha) A.alpha[t] = __fdiv_rn((float)d.w, 255.f);
            if (d.w < 255u) amin = min(amin, (uint32_t)d.w);  // floor(saturate(a) * 255 + 0.5) of a = w / 255
        }
        double er = 1.0, eg = 1.0, eb = 1.0;
        if (A.em) {
            const uchar4 e = A.em[t];
            er = lin[e.x]; eg = lin[e.y]; eb = lin[e.z];
        }
        const double emax = fmax(er, fmax(eg, eb));
        A.out1[t] = emax > 0.0 ? make_float4(unorm8(er / emax), unorm8(eg / emax), unorm8(eb / emax), one)
                               : make_float4(0.f, 0.f, 0.f, one);  // 0/0 saturates to 0
        const uchar4 m = A.mr ? A.mr[t] : make_uchar4(255, 255, 255, 255);
        A.out2[t] = make_float4(__fdiv_rn((float)m.z, 255.f), __fdiv_rn((float)m.y, 255.f), one, one);
        A.out3[t] = make_float4(one, one, one, one);
    }
    if (A.min_alpha) {
        for (int o = 16; o > 0; o >>= 1) amin = min(amin, __shfl_xor_sync(0xffffffffu, amin, o));
        if ((threadIdx.x & 31u) == 0 && amin < 255u) atomicMin(A.min_alpha, amin);
    }
}

}  // namespace

extern "C" int s2_repack_metallic_roughness(S2Context* ctx, uint32_t width, uint32_t height, const uint8_t* base_rgba8,
                                            const uint8_t* metallic_roughness_rgba8, const uint8_t* emission_rgba8,
                                            float* const* packed, float* alpha_mask, uint32_t* min_alpha,
                                            int on_device) {
    if (!ctx) return S2_ERR_INVALID;
    if (!packed || !packed[0] || !packed[1] || !packed[2] || !packed[3] || !min_alpha)
        return set_error(ctx, S2_ERR_INVALID, "the four packed images and min_alpha are required");
    if (!base_rgba8 && !metallic_roughness_rgba8 && !emission_rgba8)
        return set_error(ctx, S2_ERR_INVALID, "at least one source texture is required");
    if (alpha_mask && !base_rgba8) return set_error(ctx, S2_ERR_INVALID, "the alpha mask needs the base colour texture");
    if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28))
        return set_error(ctx, S2_ERR_INVALID, "invalid extent");
    if (on_device) {
        for (const void* p : {(const void*)base_rgba8, (const void*)metallic_roughness_rgba8, (const void*)emission_rgba8})
            if ((uintptr_t)p & 3u) return set_error(ctx, S2_ERR_INVALID, "device source textures must be 4-byte aligned");
        for (const void* p : {(const void*)packed[0], (const void*)packed[1], (const void*)packed[2], (const void*)packed[3]})
            if ((uintptr_t)p & 15u) return set_error(ctx, S2_ERR_INVALID, "device packed images must be 16-byte aligned");
        if ((uintptr_t)alpha_mask & 3u) return set_error(ctx, S2_ERR_INVALID, "the device alpha mask must be 4-byte aligned");
    }
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)width * height;
    const uint8_t* src[3] = {base_rgba8, metallic_roughness_rgba8, emission_rgba8};
    float* out[4] = {packed[0], packed[1], packed[2], packed[3]};
    float* alpha = alpha_mask;
    uint32_t* amin = nullptr;
    // device staging: inputs and outputs for host callers, the min-alpha word always
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t bytes = 256;
    if (!on_device) bytes += 3 * up(n * 4) + 4 * up(n * 16) + up(n * 4);
    char* stage = nullptr;
    int rc = check_cuda(ctx, cudaMallocAsync((void**)&stage, bytes, s), "repack staging allocation");
    if (rc != S2_OK) return rc;
    amin = (uint32_t*)stage;
    RepackArgs A{};
    A.n = (uint32_t)n;
    if (!on_device) {
        char* p = stage + 256;
        const uchar4* dsrc[3] = {nullptr, nullptr, nullptr};
        for (int k = 0; k < 3; ++k, p += up(n * 4)) {
            if (!src[k]) continue;
            cudaMemcpyAsync(p, src[k], n * 4, cudaMemcpyHostToDevice, s);
            dsrc[k] = (const uchar4*)p;
        }
        A.base = dsrc[0]; A.mr = dsrc[1]; A.em = dsrc[2];
        float4* o[4];
        for (int k = 0; k < 4; ++k, p += up(n * 16)) o[k] = (float4*)p;
        A.out0 = o[0]; A.out1 = o[1]; A.out2 = o[2]; A.out3 = o[3];
        A.alpha = alpha ? (float*)p : nullptr;
    } else {
        A.base = (const uchar4*)src[0]; A.mr = (const uchar4*)src[1]; A.em = (const uchar4*)src[2];
        A.out0 = (float4*)out[0]; A.out1 = (float4*)out[1]; A.out2 = (float4*)out[2]; A.out3 = (float4*)out[3];
        A.alpha = alpha;
    }
    A.min_alpha = base_rgba8 ? amin : nullptr;
    cudaMemsetAsync(amin, 0xff, sizeof(uint32_t), s);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + kRepackBlock - 1) / kRepackBlock, (size_t)sms * 8);
    k_repack_gltf_pbr<<<blocks, kRepackBlock, 0, s>>>(A);
    rc = check_cuda(ctx, cudaGetLastError(), "repack launch");
    uint32_t mv = 0xffffffffu;
    if (rc == S2_OK) {
        if (!on_device) {
            const float4* o[4] = {A.out0, A.out1, A.out2, A.out3};
            for (int k = 0; k < 4; ++k) cudaMemcpyAsync(out[k], o[k], n * 16, cudaMemcpyDeviceToHost, s);
            if (alpha) cudaMemcpyAsync(alpha, A.alpha, n * 4, cudaMemcpyDeviceToHost, s);
        }
        cudaMemcpyAsync(&mv, amin, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    }
    cudaFreeAsync(stage, s);
    const int sync = check_cuda(ctx, cudaStreamSynchronize(s), "repack");
    if (rc != S2_OK) return rc;
    if (sync != S2_OK) return sync;
    *min_alpha = mv == 0xffffffffu ? 255u : mv;
    return S2_OK;
}
