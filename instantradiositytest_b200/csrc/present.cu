// present.cu — the presentation pass (present.wgsl:1-8 into the
// Rgba8UnormSrgb display target of src/renderer.rs:1300-1306): every pixel
// of the filtered HDR image, clamped to [0, 1], sRGB-encoded and rounded to
// 8 bits; alpha 255.  The reference samples the HDR texel of the same pixel
// (a full-screen triangle, uv * dimensions), so there is no resampling.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace {

// IEC 61966-2-1 sRGB encoding of a linear value in [0, 1].
__device__ __forceinline__ uint32_t srgb8(float v) {
    v = fminf(fmaxf(v, 0.f), 1.f);  // also maps NaN to 0
    float e = v <= .0031308f ? v * 12.92f : 1.055f * powf(v, 1.f / 2.4f) - .055f;
    return (uint32_t)__float2int_rn(e * 255.f);
}

template <bool F16>
__global__ void __launch_bounds__(256) present_kernel(const void* __restrict__ radiance, size_t n,
                                                      uint32_t* __restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r, g, b;
    if (F16) {
        uint2 v = reinterpret_cast<const uint2*>(radiance)[i];
        __half2 a = *reinterpret_cast<__half2*>(&v.x);
        r = __low2float(a);
        g = __high2float(a);
        b = __half2float(__ushort_as_half((unsigned short)(v.y & 0xffffu)));
    } else {
        float4 v = reinterpret_cast<const float4*>(radiance)[i];
        r = v.x;
        g = v.y;
        b = v.z;
    }
    out[i] = srgb8(r) | (srgb8(g) << 8) | (srgb8(b) << 16) | (255u << 24);
}

}  // namespace

extern "C" irt_status irt_present(const void* radiance, int32_t radiance_format, uint32_t width, uint32_t height,
                                  uint8_t* rgba8, void* stream) {
    if (!radiance || !rgba8 || width == 0 || height == 0 ||
        (radiance_format != IRT_RADIANCE_F32 && radiance_format != IRT_RADIANCE_F16))
        return IRT_E_INVALID;
    const size_t n = (size_t)width * height;
    const unsigned grid = (unsigned)((n + 255) / 256);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (radiance_format == IRT_RADIANCE_F16)
        present_kernel<true><<<grid, 256, 0, st>>>(radiance, n, reinterpret_cast<uint32_t*>(rgba8));
    else
        present_kernel<false><<<grid, 256, 0, st>>>(radiance, n, reinterpret_cast<uint32_t*>(rgba8));
    return cudaGetLastError() == cudaSuccess ? IRT_OK : IRT_E_CUDA;
}
