// leafcache.cu — builds the march's leaf-order cache on the GPU.
//
// The cache is a kGridRes^3 grid over the root box of the BVH.  Per cell it
// keeps the kCellEntries objects with the smallest lower bound on their
// distance over the cell, sorted, plus the next bound as a sentinel.  A
// bound is the larger of
//   * the box bound: distance from the cell (grown by a rounding margin) to
//     the object's BVH leaf box, x 0.9998 — the walk's own pruning bound;
//   * the corner bound: the smallest object distance at the cell's eight
//     corners minus the cell's half diagonal and a margin, when all eight
//     are positive.  Positive object distances are 1-Lipschitz in world
//     space (signed box and sphere distances are; the field term is scaled by
//     the reciprocal of its trilinear gradient bound, its Pythagorean
//     extension keeps that, and the object scale and 0.9999 factor do not
//     raise it), so no point of the cell lies closer.
// The march visits a cell's objects in this order and stops at the first
// bound above its best distance; every object it skips has a distance above
// that best, so the minimum, the closest object and its voxel are those of
// the reference walk.  Corner distances use the same device code as the
// march (object_distance on the staged records and the SDF texture).
#include <cuda_runtime.h>

#include "dev_sdf.cuh"
#include "kernels.h"

namespace irtd {

struct CacheGrid {
    double org[3], size[3];
    double margin, half_diag;
};

__device__ __forceinline__ float object_distance_global(const DevScene& sc, V3 p, const MObj* objs, uint32_t o) {
    const float4* r = reinterpret_cast<const float4*>(objs + o);
    DMesh m;
    m.lo = __ldg(r + 4);
    m.hi = __ldg(r + 5);
    m.field = __ldg(reinterpret_cast<const uint4*>(r + 6));
    m.grid = __ldg(r + 7);
    m.glo = __ldg(r + 8);
    m.ghi = __ldg(r + 9);
    m.sphere = __ldg(r + 10);
    return object_distance_rows(sc, p, __ldg(r), __ldg(r + 1), __ldg(r + 2), __ldg(r + 3).x, m);
}

// Object distance at every grid corner: D[corner * n + object].
__global__ void corner_distance_kernel(const DevScene sc, const MObj* objs, uint32_t n, const CacheGrid g,
                                       float* D) {
    const uint32_t R = kGridRes + 1;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)R * R * R * n) return;
    uint32_t o = (uint32_t)(i % n);
    uint32_t c = (uint32_t)(i / n);
    uint32_t x = c % R, y = (c / R) % R, z = c / (R * R);
    V3 p = V3{(float)(g.org[0] + x * g.size[0]), (float)(g.org[1] + y * g.size[1]), (float)(g.org[2] + z * g.size[2])};
    D[i] = object_distance_global(sc, p, objs, o);
}

__global__ void cell_build_kernel(const MNode* nodes, const MObj* objs, uint32_t n, const CacheGrid g,
                                  const float* D, int use_corners, uint32_t* cells) {
    const uint32_t G = kGridRes, R = kGridRes + 1;
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= G * G * G) return;
    uint32_t ix = c % G, iy = (c / G) % G, iz = c / (G * G);
    double clo[3] = {g.org[0] + ix * g.size[0] - g.margin, g.org[1] + iy * g.size[1] - g.margin,
                     g.org[2] + iz * g.size[2] - g.margin};
    double chi[3] = {g.org[0] + (ix + 1) * g.size[0] + g.margin, g.org[1] + (iy + 1) * g.size[1] + g.margin,
                     g.org[2] + (iz + 1) * g.size[2] + g.margin};
    // the K+1 smallest (bound, object) pairs, ascending
    float best_lb[kCellEntries + 1];
    uint32_t best_id[kCellEntries + 1];
    for (uint32_t k = 0; k <= kCellEntries; k++) {
        best_lb[k] = INFINITY;
        best_id[k] = 0xffffu;
    }
    for (uint32_t o = 0; o < n; o++) {
        const uint32_t leaf = __float_as_uint(objs[o].meta.w);
        const float4 a = nodes[leaf].a, b = nodes[leaf].b;
        const double blo[3] = {a.x, a.y, a.z}, bhi[3] = {b.x, b.y, b.z};
        double s = 0.0;
        for (int k = 0; k < 3; k++) {
            double gap = fmax(0.0, fmax(blo[k] - chi[k], clo[k] - bhi[k]));
            s += gap * gap;
        }
        double lb = sqrt(s) * 0.9998 * (1.0 - 1e-6);
        if (use_corners) {
            double mn = INFINITY;
            for (uint32_t k = 0; k < 8; k++) {
                uint32_t cx = ix + (k & 1), cy = iy + ((k >> 1) & 1), cz = iz + (k >> 2);
                mn = fmin(mn, (double)D[(size_t)((cz * R + cy) * R + cx) * n + o]);
            }
            if (mn > 0.0) {
                double cb = mn - g.half_diag - 1e-3 * g.half_diag - 1e-4 - 1e-4 * mn;
                lb = fmax(lb, cb);
            }
        }
        float lbf = __double2float_rd(lb);
        if (lbf < best_lb[kCellEntries] || (lbf == best_lb[kCellEntries] && o < best_id[kCellEntries])) {
            // insert, keeping (bound, id) ascending
            int k = (int)kCellEntries;
            while (k > 0 && (best_lb[k - 1] > lbf || (best_lb[k - 1] == lbf && best_id[k - 1] > o))) {
                best_lb[k] = best_lb[k - 1];
                best_id[k] = best_id[k - 1];
                k--;
            }
            best_lb[k] = lbf;
            best_id[k] = o;
        }
    }
    uint32_t* w = cells + (size_t)c * kCellWords;
    uint32_t idw[4] = {0, 0, 0, 0};
    for (uint32_t k = 0; k < kCellEntries; k++) idw[k >> 1] |= (best_id[k] & 0xffffu) << ((k & 1) * 16);
    for (uint32_t k = 0; k < 4; k++) w[k] = idw[k];
    for (uint32_t k = 0; k < kCellEntries; k++) w[4 + k] = __float_as_uint(best_lb[k]);
    w[12] = __float_as_uint(best_lb[kCellEntries]);
    w[13] = w[14] = w[15] = 0u;
}

}  // namespace irtd

cudaError_t irt_launch_leaf_cache(const LeafCacheLaunch& L, cudaStream_t st) {
    using namespace irtd;
    CacheGrid g;
    double maxsize = 0;
    for (int a = 0; a < 3; a++) {
        g.org[a] = L.grid_org_d[a];
        g.size[a] = L.grid_size_d[a];
        maxsize = fmax(maxsize, g.size[a]);
    }
    // A point is filed by f32 arithmetic; growing each cell by this margin
    // keeps the point inside the cell box its bounds are computed for.
    g.margin = 1e-4 + 1e-5 * maxsize * kGridRes;
    double d2 = 0;
    for (int a = 0; a < 3; a++) d2 += (g.size[a] + 2 * g.margin) * (g.size[a] + 2 * g.margin);
    g.half_diag = 0.5 * sqrt(d2);
    DevScene sc{};
    sc.atlas = L.atlas;
    sc.sdf_f16 = L.sdf_f16;
    sc.sdf_cells = L.sdf_cells;
    sc.filter = L.field_filter;
    const MObj* objs = reinterpret_cast<const MObj*>(L.march_scene + 2 * (2 * L.n - 1));
    const MNode* nodes = reinterpret_cast<const MNode*>(L.march_scene);
    const int use_corners = L.corners != nullptr;
    if (use_corners) {
        const uint64_t R = kGridRes + 1;
        uint64_t total = R * R * R * L.n;
        corner_distance_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(sc, objs, L.n, g, L.corners);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const uint32_t cells = kGridRes * kGridRes * kGridRes;
    cell_build_kernel<<<(cells + 127) / 128, 128, 0, st>>>(nodes, objs, L.n, g, L.corners, use_corners, L.cells);
    return cudaGetLastError();
}
