// gbuffer.cu — CUDA G-buffer producer: one primary ray per pixel centre
// against the workload's primitives (analytic boxes and spheres, or the
// triangle hierarchies of a loaded scene with back faces culled), standing in
// for the gbuffer.wgsl raster; same outputs as irt_workload_gbuffer_cpu, in f32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <vector>

#include "dev_prims.cuh"
#include "kernels.h"
#include "workload.h"

namespace {

using irt::GPrim;

__device__ __forceinline__ void xf(const float* m, float x, float y, float z, float w, float o[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

__device__ __forceinline__ uint16_t hbits(float v) { return __half_as_ushort(__float2half_rn(v)); }

__device__ __forceinline__ uint32_t oct_snorm16(float x, float y, float z) {
    float s = fabsf(x) + fabsf(y) + fabsf(z);
    float u = x / s, v = y / s;
    if (z < 0.f) {
        float ou = (1.f - fabsf(v)) * (u >= 0.f ? 1.f : -1.f);
        float ov = (1.f - fabsf(u)) * (v >= 0.f ? 1.f : -1.f);
        u = ou;
        v = ov;
    }
    int qu = __float2int_rn(fminf(fmaxf(u, -1.f), 1.f) * 32767.f);
    int qv = __float2int_rn(fminf(fmaxf(v, -1.f), 1.f) * 32767.f);
    return ((uint32_t)(uint16_t)(int16_t)qu) | ((uint32_t)(uint16_t)(int16_t)qv << 16);
}

__global__ void gbuffer_kernel(const __grid_constant__ irt_frame f, const irt::PrimTable T, int fmt,
                               float* depth, void* normal, void* color, void* params, void* motion) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    uint32_t W = f.size[0], H = f.size[1];
    if (x >= W || y >= H) return;
    size_t i = (size_t)y * W + x;
    float u = ((float)x + .5f) / (float)W, v = ((float)y + .5f) / (float)H;
    float nx = u * 2.f - 1.f, ny = 1.f - v * 2.f;
    float pn[4], pf[4];
    xf(f.inv_vp.m, nx, ny, 0.f, 1.f, pn);
    xf(f.inv_vp.m, nx, ny, 1.f, 1.f, pf);
    float o[3] = {pn[0] / pn[3], pn[1] / pn[3], pn[2] / pn[3]};
    float d[3] = {pf[0] / pf[3] - o[0], pf[1] / pf[3] - o[1], pf[2] / pf[3] - o[2]};
    // d spans near to far plane: t in [0, 1).
    float best;
    float nl_best[3] = {0, 0, 0};
    int hit = irtd::cast_prims(T, o, d, 0.f, 1.f, true, best, nl_best);
    float dep = 1.f, nrm[3] = {0, 0, 0}, col[3] = {0, 0, 0}, par[2] = {0, 0}, mot[2] = {0, 0};
    if (hit >= 0) {
        const GPrim& p = T.prims[hit];
        float w[4];
        xf(p.model, nl_best[0], nl_best[1], nl_best[2], 0.f, w);
        float inv = 1.f / sqrtf(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        nrm[0] = w[0] * inv;
        nrm[1] = w[1] * inv;
        nrm[2] = w[2] * inv;
        float P[3] = {o[0] + d[0] * best, o[1] + d[1] * best, o[2] + d[2] * best};
        float c[4], pc[4];
        xf(f.vp.m, P[0], P[1], P[2], 1.f, c);
        xf(f.previous_vp.m, P[0], P[1], P[2], 1.f, pc);
        dep = fminf(c[2] / c[3], 0.99999994f);
        col[0] = p.color[0];
        col[1] = p.color[1];
        col[2] = p.color[2];
        par[0] = p.params[0];
        par[1] = p.params[1];
        mot[0] = (c[0] / c[3] - pc[0] / pc[3]) * .5f;
        mot[1] = (c[1] / c[3] - pc[1] / pc[3]) * -.5f;
    }
    float alpha = hit >= 0 ? 1.f : 0.f;
    depth[i] = dep;
    if (fmt == IRT_GBUFFER_F32) {
        ((float4*)normal)[i] = make_float4(nrm[0], nrm[1], nrm[2], alpha);
        ((float4*)color)[i] = make_float4(col[0], col[1], col[2], alpha);
        ((float2*)params)[i] = make_float2(par[0], par[1]);
        ((float2*)motion)[i] = make_float2(mot[0], mot[1]);
    } else if (fmt == IRT_GBUFFER_F16) {
        ((uint2*)normal)[i] = make_uint2(hbits(nrm[0]) | ((uint32_t)hbits(nrm[1]) << 16), hbits(nrm[2]) | ((uint32_t)hbits(alpha) << 16));
        ((uint2*)color)[i] = make_uint2(hbits(col[0]) | ((uint32_t)hbits(col[1]) << 16), hbits(col[2]) | ((uint32_t)hbits(alpha) << 16));
        ((uint32_t*)params)[i] = hbits(par[0]) | ((uint32_t)hbits(par[1]) << 16);
        ((uint32_t*)motion)[i] = hbits(mot[0]) | ((uint32_t)hbits(mot[1]) << 16);
    } else {
        ((uint32_t*)normal)[i] = hit >= 0 ? oct_snorm16(nrm[0], nrm[1], nrm[2]) : 0u;
        auto q8 = [](float c) { return (uint32_t)__float2int_rn(fminf(fmaxf(c, 0.f), 1.f) * 255.f); };
        ((uint32_t*)color)[i] = q8(col[0]) | (q8(col[1]) << 8) | (q8(col[2]) << 16) | (q8(alpha) << 24);
        ((uint32_t*)params)[i] = hbits(par[0]) | ((uint32_t)hbits(par[1]) << 16);
        ((uint32_t*)motion)[i] = hbits(mot[0]) | ((uint32_t)hbits(mot[1]) << 16);
    }
}

}  // namespace

// Flattened primitive table of a workload on the current device (static
// scenes: built once and kept with the workload), with the triangle
// hierarchies of loaded meshes concatenated into shared node and triangle
// tables.
// Frees a workload's device primitive tables (Workload::release_device).
static void release_prims(irt::Workload& w) {
    int prev = -1;
    cudaGetDevice(&prev);
    const bool other = w.dev_prims_device >= 0 && prev != w.dev_prims_device;
    if (other) cudaSetDevice(w.dev_prims_device);
    for (void* p : {w.dev_prims, w.dev_nodes, w.dev_tris})
        if (p) cudaFree(p);
    w.dev_prims = w.dev_nodes = w.dev_tris = nullptr;
    if (other && prev >= 0) cudaSetDevice(prev);
}

cudaError_t irt_workload_prims(const irt_workload* wl_c, irt::PrimTable* out) {
    irt_workload* wl = const_cast<irt_workload*>(wl_c);
    irt::Workload& w = wl->w;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!w.dev_prims || w.dev_prims_device != dev) {
        std::vector<GPrim> prims;
        std::vector<irt::TriNode> nodes;
        std::vector<irt::TriRec> tris;
        std::vector<uint32_t> node_base(w.mesh_desc.size(), 0), tri_base(w.mesh_desc.size(), 0);
        for (size_t m = 0; m < w.mesh_desc.size(); m++) {
            const irt::MeshDesc& md = w.mesh_desc[m];
            if (!md.triangles) continue;
            node_base[m] = (uint32_t)nodes.size();
            tri_base[m] = (uint32_t)tris.size();
            nodes.insert(nodes.end(), md.bvh.nodes.begin(), md.bvh.nodes.end());
            tris.insert(tris.end(), md.bvh.tris.begin(), md.bvh.tris.end());
        }
        for (uint32_t oi = 0; oi < w.objs.size(); oi++) {
            const irt::Obj& ob = w.objs[oi];
            irt_mat4 model = irt::to_f32(ob.model), inv = irt::to_f32(ob.inv_model);
            const irt_material& m = w.materials[ob.material];
            const irt::MeshDesc& md = w.mesh_desc[ob.mesh];
            GPrim g{};
            for (int k = 0; k < 16; k++) {
                g.inv_model[k] = inv.m[k];
                g.model[k] = model.m[k];
            }
            for (int k = 0; k < 3; k++) g.color[k] = m.color[k];
            g.params[0] = fminf(fmaxf(m.params[0], .045f), 1.f);
            g.params[1] = fminf(fmaxf(m.params[1], 0.f), 1.f);
            g.object = oi;
            if (md.triangles) {
                if (md.bvh.nodes.empty()) continue;
                g.kind = irt::kPrimTriangles;
                for (int a = 0; a < 3; a++) {
                    g.lo[a] = md.bvh.nodes[0].lo[a];
                    g.hi[a] = md.bvh.nodes[0].hi[a];
                }
                g.node_base = node_base[ob.mesh];
                g.tri_base = tri_base[ob.mesh];
                prims.push_back(g);
                continue;
            }
            for (const irt::Part& part : md.parts) {
                for (int a = 0; a < 3; a++) {
                    g.lo[a] = part.sphere ? 0.f : (float)part.lo[a];
                    g.hi[a] = part.sphere ? 0.f : (float)part.hi[a];
                }
                if (part.sphere) g.lo[0] = (float)part.radius;
                g.kind = part.sphere ? irt::kPrimSphere : irt::kPrimBox;
                prims.push_back(g);
            }
        }
        for (void** p : {&w.dev_prims, &w.dev_nodes, &w.dev_tris}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        w.dev_prims_count = 0;
        w.release_device = &release_prims;
        auto upload = [](void** dst, const void* src, size_t bytes) {
            if (bytes == 0) return cudaSuccess;
            cudaError_t r = cudaMalloc(dst, bytes);
            if (r != cudaSuccess) return r;
            return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        };
        e = upload(&w.dev_prims, prims.data(), prims.size() * sizeof(GPrim));
        if (e == cudaSuccess) e = upload(&w.dev_nodes, nodes.data(), nodes.size() * sizeof(irt::TriNode));
        if (e == cudaSuccess) e = upload(&w.dev_tris, tris.data(), tris.size() * sizeof(irt::TriRec));
        if (e != cudaSuccess) return e;
        w.dev_prims_device = dev;
        w.dev_prims_count = (uint32_t)prims.size();
    }
    out->prims = static_cast<const GPrim*>(w.dev_prims);
    out->n = w.dev_prims_count;
    out->nodes = static_cast<const irt::TriNode*>(w.dev_nodes);
    out->tris = static_cast<const irt::TriRec*>(w.dev_tris);
    return cudaSuccess;
}

extern "C" irt_status irt_gbuffer_render(irt_context* ctx, const irt_workload* wl, const irt_frame* f,
                                         const irt_object* objects, int32_t format, float* depth, void* normal,
                                         void* color, void* params, void* motion, void* stream) {
    (void)objects;
    if (!ctx || !wl || !f || !depth || !normal || !color || !params || !motion) return IRT_E_INVALID;
    if (format < IRT_GBUFFER_F32 || format > IRT_GBUFFER_PACKED) return IRT_E_INVALID;
    irt::PrimTable T{};
    if (irt_workload_prims(wl, &T) != cudaSuccess) return IRT_E_CUDA;
    dim3 block(32, 8);
    dim3 grid((f->size[0] + 31) / 32, (f->size[1] + 7) / 8);
    gbuffer_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        *f, T, format, depth, normal, color, params, motion);
    return cudaGetLastError() == cudaSuccess ? IRT_OK : IRT_E_CUDA;
}
