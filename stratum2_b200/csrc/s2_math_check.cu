// s2_device_math: evaluates the path tracer's device math functions (the RNG, octahedral normal
// packing, microfacet helpers and sampling maps of s2_math.cuh / s2_bsdf.cuh) on caller-given
// inputs, so that they can be checked one at a time against the reference's own shader functions
// (src/Shaders/common/rng.hlsli, common.hlsli, microfacet.hlsli).  A diagnostic entry point: the
// renderers call these functions inline.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "s2_bsdf.cuh"
#include "s2_context.h"

namespace {

constexpr int kIn = 8, kOut = 9;  // doubles per entry, as in the header

__global__ void k_device_math(int fn, const double* __restrict__ in, uint32_t n, double* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double* a = in + (size_t)kIn * k;
    double* o = out + (size_t)kOut * k;
    auto f = [&](int i) { return (float)a[i]; };
    auto u = [&](int i) { return (uint32_t)a[i]; };
    auto put3 = [&](float3 v, int at) { o[at] = v.x; o[at + 1] = v.y; o[at + 2] = v.z; };
    switch (fn) {
        case 0: o[0] = xxhash32(u(0)); break;
        case 1: o[0] = pcg_hash(u(0)); break;
        case 2: { const uint4 r = pcg4d(make_uint4(u(0), u(1), u(2), u(3))); o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w; break; }
        case 3: {
            Rng rng = make_rng(u(0), u(1), u(2), false);
            rng.ctr = u(3);
            const float4 r = rng.next_float();
            o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
            break;
        }
        case 4: o[0] = pack_normal(f3(f(0), f(1), f(2))); break;
        case 5: put3(unpack_normal(u(0)), 0); break;
        case 6: o[0] = gtr1(f(0), f(1)); break;
        case 7: o[0] = gtr2(f3(f(0), f(1), f(2)), f(3), f(4)); break;
        case 8: o[0] = smith_gtr2(f3(f(0), f(1), f(2)), f(3), f(4)); break;
        case 9: o[0] = smith_gtr1(f3(f(0), f(1), f(2))); break;
        case 10: put3(sample_vndf(f3(f(0), f(1), f(2)), f(3), f(4), f(5), f(6)), 0); break;
        case 11: o[0] = schlick1(f(0), f(1)); break;
        case 12: o[0] = fresnel_dielectric(f(0), f(1)); break;
        case 13: { const float2 r = sample_concentric_disc(f(0), f(1)); o[0] = r.x; o[1] = r.y; break; }
        case 14: put3(sample_cos_hemisphere(f(0), f(1)), 0); break;
        case 15: put3(sample_uniform_sphere(f(0), f(1)), 0); break;
        case 16: { const float2 r = sample_uniform_triangle(f(0), f(1)); o[0] = r.x; o[1] = r.y; break; }
        case 17: {
            const float3 nn = f3(f(0), f(1), f(2));
            float3 t, b;
            make_orthonormal(nn, t, b);
            put3(t, 0); put3(b, 3); put3(nn, 6);
            break;
        }
    }
}

}  // namespace

extern "C" int s2_device_math(S2Context* ctx, int fn, const double* in, uint32_t n, double* out) {
    if (!ctx) return S2_ERR_INVALID;
    if (fn < 0 || fn > 17) return s2::set_error(ctx, S2_ERR_INVALID, "s2_device_math: unknown function id");
    if (n == 0) return S2_OK;
    if (!in || !out) return s2::set_error(ctx, S2_ERR_INVALID, "s2_device_math: null input or output");
    cudaSetDevice(ctx->device);
    std::vector<s2::DevBuf> tmp;
    double* din = (double*)s2::dev_alloc(ctx, tmp, sizeof(double) * kIn * (size_t)n);
    double* dout = (double*)s2::dev_alloc(ctx, tmp, sizeof(double) * kOut * (size_t)n);
    if (!din || !dout) { s2::free_bufs(tmp); return S2_ERR_OOM; }
    cudaMemcpyAsync(din, in, sizeof(double) * kIn * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(dout, 0, sizeof(double) * kOut * (size_t)n, ctx->stream);
    k_device_math<<<(n + 127) / 128, 128, 0, ctx->stream>>>(fn, din, n, dout);
    int rc = s2::check_cuda(ctx, cudaGetLastError(), "s2_device_math launch");
    if (rc == S2_OK) {
        cudaMemcpyAsync(out, dout, sizeof(double) * kOut * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        rc = s2::check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "s2_device_math");
    }
    s2::free_bufs(tmp);
    return rc;
}
