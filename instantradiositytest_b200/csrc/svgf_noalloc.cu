// svgf_noalloc.cu — the SVGF spatial stages (variance bootstrap and the
// a-trous wavelets) for callers that cannot allocate device memory.
//
// Some hosts never let a library call cudaMalloc: a renderer whose frame
// thread must not stall on the device-wide synchronisation an allocation can
// imply, or an application that reserves all device memory up front under
// its own allocator and budget.  This entry point serves them: the caller
// passes every input and output, and what the filter needs in between — the
// per-pixel positions and edge-stopping features of the frame and the two
// ping-pong images of the a-trous passes — lives in a fixed array of this
// library's device memory instead of a session.
//
// The array (kNoAllocMaxPixels x 5 f32x4 texels = 20 MiB) is a file-scope
// __device__ variable: every GPU that loads the library holds it until the
// process exits.  Frames above kNoAllocMaxPixels pixels are rejected.  All
// calls share the array and it keeps the last call's contents (each call
// rewrites every texel it reads before reading it), so calls that overlap on
// the GPU (on different streams, or from different host threads without
// ordering) race on it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "kernels.h"

namespace {

constexpr uint32_t kNoAllocMaxPixels = 512u * 512u;
constexpr int kMaxDevices = 64;

// Per pixel: [0] ping and [1] pong a-trous images (f32x4; f16x4 images use
// the first half of each), [2] world position + SVGF pixel scale, [3..4]
// edge-stopping feature records (two f32x4 per pixel, decoded G-buffer
// formats only).
static __device__ __align__(256) float4 g_svgf_scratch[5][kNoAllocMaxPixels];

// Device address of g_svgf_scratch per device ordinal, looked up on the first
// call on that device.  In host code the symbol itself is only a host-side
// stand-in, never a device address.  The cached address belongs to the
// device's primary context: a caller that resets the device
// (cudaDeviceReset) while the library stays loaded must not call this entry
// point again in that process.
std::mutex g_mu;
float4* g_scratch_ptr[kMaxDevices] = {};

void fail(char* err, size_t err_len, const char* msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
}

}  // namespace

extern "C" irt_status irt_svgf_spatial_noalloc(const irt_frame* frame, const irt_gbuffer* gbuffer,
                                               int32_t radiance_format, int32_t moments_format,
                                               uint32_t iterations, const void* temporal_radiance,
                                               const void* moments, void* filtered_out, void* feedback_out,
                                               void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = 0;
    if (!frame || !gbuffer || !temporal_radiance || !moments || !filtered_out) {
        fail(err, err_len, "null argument");
        return IRT_E_INVALID;
    }
    const uint64_t pixels = (uint64_t)frame->size[0] * frame->size[1];
    if (pixels == 0 || pixels > kNoAllocMaxPixels) {
        fail(err, err_len, "frame exceeds the allocation-free filter's maximum of 262144 pixels (512x512)");
        return IRT_E_INVALID;
    }
    if (iterations == 0 || iterations > 5) {
        fail(err, err_len, "svgf iterations must be 1..5");
        return IRT_E_INVALID;
    }
    if (radiance_format != IRT_RADIANCE_F32 && radiance_format != IRT_RADIANCE_F16) {
        fail(err, err_len, "unknown radiance format");
        return IRT_E_INVALID;
    }
    if (moments_format != IRT_MOMENTS_F32 && moments_format != IRT_MOMENTS_F16) {
        fail(err, err_len, "unknown moments format");
        return IRT_E_INVALID;
    }
    if (gbuffer->format < IRT_GBUFFER_F32 || gbuffer->format > IRT_GBUFFER_PACKED || !gbuffer->depth ||
        !gbuffer->normal || !gbuffer->color || !gbuffer->params || !gbuffer->motion) {
        fail(err, err_len, "invalid G-buffer format or planes");
        return IRT_E_INVALID;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        fail(err, err_len, "no usable current CUDA device");
        return IRT_E_NODEVICE;
    }
    float4* scratch = nullptr;
    {
        // Set-up on the first call on each device, with that device current.
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_svgf_scratch);
            if (e != cudaSuccess || !p) {
                fail(err, err_len, cudaGetErrorString(e));
                return IRT_E_CUDA;
            }
            g_scratch_ptr[dev] = static_cast<float4*>(p);
        }
        scratch = g_scratch_ptr[dev];
    }
    float4* ping = scratch;
    float4* pong = scratch + kNoAllocMaxPixels;
    float4* guide = scratch + 2 * kNoAllocMaxPixels;
    float4* feat = scratch + 3 * kNoAllocMaxPixels;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SvgfLaunch L{};
    L.frame = frame;
    L.gbuffer = *gbuffer;
    L.radiance_f16 = radiance_format == IRT_RADIANCE_F16;
    L.moments_f16 = moments_format == IRT_MOMENTS_F16;
    // The frame's per-pixel positions (and, for the F16 and packed G-buffers,
    // decoded edge-stopping features), written by the same kernels a session
    // runs before its SVGF passes, so the results equal a session's.
    L.out = guide;
    L.out2 = feat;
    cudaError_t e = irt_launch_svgf(L, gbuffer->format == IRT_GBUFFER_F32 ? 3 : 6, st);
    L.guide = guide;
    L.feat = feat;
    // svgf_variance (svgf.wgsl:77-89): temporal radiance + moments -> ping.
    L.in = temporal_radiance;
    L.moments_in = moments;
    L.out = ping;
    L.out2 = nullptr;
    if (e == cudaSuccess) e = irt_launch_svgf(L, 1, st);
    // svgf_atrous x iterations (svgf.wgsl:91-110), the same buffer order as a
    // session: iteration 0 also gives the feedback image, the last writes
    // filtered_out, the others alternate between pong and ping.
    const void* in = ping;
    for (uint32_t i = 0; i < iterations && e == cudaSuccess; i++) {
        void* out = (i + 1 == iterations) ? filtered_out : (i % 2 == 0 ? (void*)pong : (void*)ping);
        L.in = in;
        L.out = out;
        L.out2 = i == 0 ? feedback_out : nullptr;
        L.step = 1 << i;
        e = irt_launch_svgf(L, 2, st);
        in = out;
    }
    if (e != cudaSuccess) {
        fail(err, err_len, cudaGetErrorString(e));
        return IRT_E_CUDA;
    }
    return IRT_OK;
}
