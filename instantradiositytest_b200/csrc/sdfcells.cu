// sdfcells.cu — corner cells of a field mesh: for each of its (res-1)^3
// cells the 8 corner texels of the atlas tile in one record, so that a
// trilinear sample (common.wgsl:31-38) reads one 32-byte (f32) or 16-byte
// (f16) record instead of 8 texture fetches.  Built once per scene from the
// atlas texture; the values are the texels themselves.  Every sample of a
// field (sample_field in dev_sdf.cuh) reads these records.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace {

__global__ void pack_cells_kernel(cudaTextureObject_t atlas, int f16, uint3 origin, uint32_t res, uint64_t base,
                                  void* out) {
    const uint32_t n = res - 1u;
    const uint64_t cells = (uint64_t)n * n * n;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cx = (uint32_t)(i % n), cy = (uint32_t)((i / n) % n), cz = (uint32_t)(i / ((uint64_t)n * n));
        const float bx = (float)(origin.x + cx) + .5f, by = (float)(origin.y + cy) + .5f,
                    bz = (float)(origin.z + cz) + .5f;
        float t[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            t[k] = tex3D<float>(atlas, bx + (float)(k & 1), by + (float)((k >> 1) & 1), bz + (float)(k >> 2));
        if (f16) {
            uint32_t w[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                w[k] = (uint32_t)__half_as_ushort(__float2half_rn(t[2 * k])) |
                       ((uint32_t)__half_as_ushort(__float2half_rn(t[2 * k + 1])) << 16);
            static_cast<uint4*>(out)[base + i] = make_uint4(w[0], w[1], w[2], w[3]);
        } else {
            float4* o = static_cast<float4*>(out) + 2 * (base + i);
            o[0] = make_float4(t[0], t[1], t[2], t[3]);
            o[1] = make_float4(t[4], t[5], t[6], t[7]);
        }
    }
}

}  // namespace

cudaError_t irt_pack_sdf_cells(cudaTextureObject_t atlas, int f16, const uint32_t origin[3], uint32_t res,
                               uint64_t base, void* out, cudaStream_t st) {
    if (res < 2) return cudaErrorInvalidValue;
    const uint64_t n = res - 1u, cells = n * n * n;
    const uint32_t blocks = (uint32_t)((cells + 255) / 256 < 148u * 16u ? (cells + 255) / 256 : 148u * 16u);
    pack_cells_kernel<<<blocks, 256, 0, st>>>(atlas, f16, make_uint3(origin[0], origin[1], origin[2]), res, base,
                                              out);
    return cudaGetLastError();
}
