// sdfcells.cu — corner cells of a field mesh: for each of its (res-1)^3
// cells the 8 corner texels of the atlas tile in one record, so that a
// trilinear sample (common.wgsl:31-38) reads one 32-byte (f32) or 16-byte
// (f16) record instead of 8 texture fetches.  Built once per scene from the
// atlas texture; the values are the texels themselves.  Every sample of a
// field (sample_field in dev_sdf.cuh) reads these records.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "dev_sdf.cuh"
#include "kernels.h"

namespace {

// sample_field of one mesh at n grid-space points with the kernels' own
// sampler (the point-sampled trilinear of the IEEE build, or the hardware
// linear fetch).
__global__ void sample_points_kernel(const irtd::DevScene sc, const irtd::DMesh m, const float* __restrict__ q,
                                     uint32_t n, float* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = irtd::sample_field(sc, m, irtd::V3{q[3 * i], q[3 * i + 1], q[3 * i + 2]});
}

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

cudaError_t irt_launch_sample_field(const irtd::DevScene& sc, const irt_mesh& row, const float* q, uint32_t n,
                                    float* out, cudaStream_t st) {
    irtd::DMesh m;
    m.lo = make_float4(row.lo[0], row.lo[1], row.lo[2], row.lo[3]);
    m.hi = make_float4(row.hi[0], row.hi[1], row.hi[2], row.hi[3]);
    m.field = make_uint4(row.field[0], row.field[1], row.field[2], row.field[3]);
    m.grid = make_float4(row.grid[0], row.grid[1], row.grid[2], row.grid[3]);
    m.glo = make_float4(row.geometry_lo[0], row.geometry_lo[1], row.geometry_lo[2], row.geometry_lo[3]);
    m.ghi = make_float4(row.geometry_hi[0], row.geometry_hi[1], row.geometry_hi[2], row.geometry_hi[3]);
    m.sphere = make_float4(row.enclosing_sphere[0], row.enclosing_sphere[1], row.enclosing_sphere[2],
                           row.enclosing_sphere[3]);
    const uint32_t blocks = (n + 255) / 256 < 148u * 8u ? (n + 255) / 256 : 148u * 8u;
    sample_points_kernel<<<blocks, 256, 0, st>>>(sc, m, q, n, out);
    return cudaGetLastError();
}

cudaError_t irt_pack_sdf_cells(cudaTextureObject_t atlas, int f16, const uint32_t origin[3], uint32_t res,
                               uint64_t base, void* out, cudaStream_t st) {
    if (res < 2) return cudaErrorInvalidValue;
    const uint64_t n = res - 1u, cells = n * n * n;
    const uint32_t blocks = (uint32_t)((cells + 255) / 256 < 148u * 16u ? (cells + 255) / 256 : 148u * 16u);
    pack_cells_kernel<<<blocks, 256, 0, st>>>(atlas, f16, make_uint3(origin[0], origin[1], origin[2]), res, base,
                                              out);
    return cudaGetLastError();
}
