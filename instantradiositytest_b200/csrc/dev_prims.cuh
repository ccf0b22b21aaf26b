// dev_prims.cuh — f32 ray casts against the flattened primitive table of a
// workload: analytic boxes and spheres of the procedural rooms, triangle
// hierarchies of loaded scene files (tri_bvh.h), all in object space.  Used by
// the CUDA G-buffer producer (primary rays) and the CUDA VPL generator (the
// stand-in for the ray query of vpl.wgsl).
#pragma once
#include <cuda_runtime.h>

#include "workload.h"

namespace irtd {

__device__ __forceinline__ void xf4(const float* m, float x, float y, float z, float w, float o[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

__device__ __forceinline__ bool slab(const float lo[3], const float hi[3], const float o[3], const float inv[3],
                                     float tmin, float tmax) {
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float t0 = (lo[a] - o[a]) * inv[a], t1 = (hi[a] - o[a]) * inv[a];
        tmin = fmaxf(tmin, fminf(t0, t1));
        tmax = fminf(tmax, fmaxf(t0, t1));
    }
    return tmin <= tmax;
}

// Nearest hit in (tmin, best) of one triangle hierarchy (Moller-Trumbore in
// f32; `cull` skips triangles whose geometric normal faces along d).  On a
// hit updates best and writes the interpolated vertex normal to nl.  The
// stack holds kTriStack entries, above the depth of any hierarchy that
// build_tri_bvh makes; a push that would not fit is dropped.
__device__ __forceinline__ bool cast_tris(const irt::TriNode* nodes, const irt::TriRec* tris, const float o[3],
                                          const float d[3], float tmin, bool cull, float& best, float nl[3]) {
    const float inv[3] = {1.f / d[0], 1.f / d[1], 1.f / d[2]};
    uint32_t stack[irt::kTriStack];
    uint32_t sp = 0;
    stack[sp++] = 0;
    int hit = -1;
    float bu = 0.f, bv = 0.f;
    while (sp) {
        const float4* np = reinterpret_cast<const float4*>(nodes + stack[--sp]);
        const float4 a = __ldg(np), b = __ldg(np + 1);
        const float lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
        if (!slab(lo, hi, o, inv, tmin, best)) continue;
        const uint32_t first = __float_as_uint(a.w), count = __float_as_uint(b.w);
        if (count == 0u) {
            if (sp + 2u > irt::kTriStack) continue;
            stack[sp++] = first + 1u;
            stack[sp++] = first;
            continue;
        }
        for (uint32_t j = first; j < first + count; j++) {
            const float4* tp = reinterpret_cast<const float4*>(tris + j);
            const float4 v0 = __ldg(tp), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2);
            if (cull) {
                const float gx = e1.y * e2.z - e1.z * e2.y, gy = e1.z * e2.x - e1.x * e2.z,
                            gz = e1.x * e2.y - e1.y * e2.x;
                if (gx * d[0] + gy * d[1] + gz * d[2] >= 0.f) continue;
            }
            const float px = d[1] * e2.z - d[2] * e2.y, py = d[2] * e2.x - d[0] * e2.z, pz = d[0] * e2.y - d[1] * e2.x;
            const float det = e1.x * px + e1.y * py + e1.z * pz;
            if (det == 0.f) continue;
            const float id = 1.f / det;
            const float sx = o[0] - v0.x, sy = o[1] - v0.y, sz = o[2] - v0.z;
            const float u = (sx * px + sy * py + sz * pz) * id;
            if (u < 0.f || u > 1.f) continue;
            const float qx = sy * e1.z - sz * e1.y, qy = sz * e1.x - sx * e1.z, qz = sx * e1.y - sy * e1.x;
            const float v = (d[0] * qx + d[1] * qy + d[2] * qz) * id;
            if (v < 0.f || u + v > 1.f) continue;
            const float t = (e2.x * qx + e2.y * qy + e2.z * qz) * id;
            if (t > tmin && t < best) {
                best = t;
                hit = (int)j;
                bu = u;
                bv = v;
            }
        }
    }
    if (hit < 0) return false;
    const float4* tp = reinterpret_cast<const float4*>(tris + hit);
    const float4 v0 = __ldg(tp), e1 = __ldg(tp + 1), e2 = __ldg(tp + 2), n1 = __ldg(tp + 3), n2 = __ldg(tp + 4);
    const float w0 = 1.f - bu - bv;
    nl[0] = v0.w * w0 + n1.x * bu + n2.x * bv;
    nl[1] = e1.w * w0 + n1.y * bu + n2.y * bv;
    nl[2] = e2.w * w0 + n1.z * bu + n2.z * bv;
    return true;
}

// Nearest hit t in (tmin, tmax) along o + t d over all primitives: front
// entries of boxes (slab test; an origin inside a box is no hit) and spheres
// (nearest root), and triangle hierarchies (back faces skipped when `cull`).
// Returns the primitive index or -1, with t and the object-space normal in
// nl (the entered face, or the interpolated vertex normal of a triangle).
__device__ __forceinline__ int cast_prims(const irt::PrimTable& T, const float o[3], const float d[3], float tmin,
                                          float tmax, bool cull, float& t_out, float nl[3]) {
    const irt::GPrim* prims = T.prims;
    float best = tmax;
    int hit = -1;
    for (uint32_t k = 0; k < T.n; k++) {
        const irt::GPrim& p = prims[k];
        float lo4[4], ld4[4];
        xf4(p.inv_model, o[0], o[1], o[2], 1.f, lo4);
        xf4(p.inv_model, d[0], d[1], d[2], 0.f, ld4);
        float t = 0.f;
        float nn[3] = {0, 0, 0};
        bool h = false;
        if (p.kind == irt::kPrimTriangles) {
            const float inv[3] = {1.f / ld4[0], 1.f / ld4[1], 1.f / ld4[2]};
            if (slab(p.lo, p.hi, lo4, inv, tmin, best) &&
                cast_tris(T.nodes + p.node_base, T.tris + p.tri_base, lo4, ld4, tmin, cull, best, nl)) {
                hit = (int)k;
            }
            continue;
        }
        if (p.kind == irt::kPrimSphere) {
            float r = p.lo[0];
            float b = lo4[0] * ld4[0] + lo4[1] * ld4[1] + lo4[2] * ld4[2];
            float a = ld4[0] * ld4[0] + ld4[1] * ld4[1] + ld4[2] * ld4[2];
            float c = lo4[0] * lo4[0] + lo4[1] * lo4[1] + lo4[2] * lo4[2] - r * r;
            float disc = b * b - a * c;
            if (disc >= 0.f) {
                t = (-b - sqrtf(disc)) / a;
                if (t >= tmin && t < best) {
                    h = true;
                    for (int q = 0; q < 3; q++) nn[q] = (lo4[q] + ld4[q] * t) / r;
                }
            }
        } else {
            float t0 = tmin, t1 = best;
            int axis = -1;
            float sign = 0.f;
            bool miss = false;
            for (int a = 0; a < 3 && !miss; a++) {
                float inv = 1.f / ld4[a];
                float ta = (p.lo[a] - lo4[a]) * inv, tb = (p.hi[a] - lo4[a]) * inv;
                float s = -1.f;
                if (ta > tb) {
                    float tmp = ta;
                    ta = tb;
                    tb = tmp;
                    s = 1.f;
                }
                if (ta > t0) {
                    t0 = ta;
                    axis = a;
                    sign = s;
                }
                t1 = fminf(t1, tb);
                if (t0 > t1) miss = true;
            }
            if (!miss && axis >= 0 && t0 < best) {
                h = true;
                t = t0;
                nn[axis] = sign;
            }
        }
        if (h) {
            best = t;
            hit = (int)k;
            nl[0] = nn[0];
            nl[1] = nn[1];
            nl[2] = nn[2];
        }
    }
    t_out = best;
    return hit;
}

}  // namespace irtd
