// dev_sdf.cuh — device restatement of sdf.wgsl: signed distance bounds of
// meshes (certified boxes exactly, others from the trilinear SDF atlas read
// through the texture path), the stackless preorder BVH walk with escape links
// and the Quilez soft-shadow march.
#pragma once
#include "dev_common.cuh"
#include "kernels.h"

namespace irtd {

struct DevScene {
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    const irt_light* lights;
    cudaTextureObject_t atlas;  // 3-D R32F or R16F texels, point sampled
    int32_t sdf_f16;            // texel = f16(value / mesh.lo[3])
    uint32_t* error;            // device error word
    // Corner cells of the field meshes, built from the atlas at scene
    // creation (sdfcells.cu): cell (cx, cy, cz) of a mesh of resolution res
    // is record bits(mesh.hi[3]) + (cz * (res-1) + cy) * (res-1) + cx,
    // holding the 8 texels t[k] at (cx + (k&1), cy + (k>>1 & 1), cz + (k>>2))
    // of its atlas tile — two float4 (f32) or eight halves in one uint4 (f16).
    const void* sdf_cells;
    FieldFilter filter;
};

// Read-only-path loads of the scene records as 16-byte vectors.
struct DMesh {
    float4 lo, hi;
    uint4 field;
    float4 grid, glo, ghi, sphere;
};
__device__ __forceinline__ DMesh load_mesh(const irt_mesh* base, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(base + i);
    DMesh m;
    m.lo = __ldg(p);
    m.hi = __ldg(p + 1);
    m.field = __ldg(reinterpret_cast<const uint4*>(p + 3));
    m.grid = __ldg(p + 4);
    m.glo = __ldg(p + 5);
    m.ghi = __ldg(p + 6);
    m.sphere = __ldg(p + 7);
    return m;
}
struct DObject {  // inverse matrix columns and info
    float4 c0, c1, c2, c3;
    uint4 info;
};
__device__ __forceinline__ DObject load_object(const irt_object* base, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(base + i);
    DObject o;
    o.c0 = __ldg(p + 8);
    o.c1 = __ldg(p + 9);
    o.c2 = __ldg(p + 10);
    o.c3 = __ldg(p + 11);
    o.info = __ldg(reinterpret_cast<const uint4*>(p + 12));
    return o;
}
struct DNode {
    float4 lo, hi;
    uint4 info;
};
__device__ __forceinline__ DNode load_node(const irt_node* base, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(base + i);
    return DNode{__ldg(p), __ldg(p + 1), __ldg(reinterpret_cast<const uint4*>(p + 2))};
}

// sdf.wgsl:1-4
__device__ __forceinline__ float signed_box_distance(V3 p, V3 lo, V3 hi) {
    V3 delta = vmax(lo - p, p - hi);
    return length(vmax(delta, V3{0.f, 0.f, 0.f})) + wmin(wmax(delta.x, wmax(delta.y, delta.z)), 0.f);
}

// common.wgsl:31-38 — the 8 texels of the cell (clamped to res-2), weights in
// z, y, x order as the WGSL loop accumulates them.
__device__ __forceinline__ float sample_field(const DevScene& sc, const DMesh& m, V3 q) {
    if (sc.filter.linear) {
        // textureSampleLevel(fields, field_sampler, (vec3<f32>(origin)+q+.5)/vec3<f32>(dims), 0.):
        // the sampler takes the texel coordinate origin + q + .5 (the
        // normalised coordinate times the extent), filters between texels
        // floor(x - .5) and the next with 8-bit fixed-point weights, and
        // clamps to the atlas edge.
        const float u = __fadd_rn(__fadd_rn((float)m.field.x, q.x), .5f);
        const float v = __fadd_rn(__fadd_rn((float)m.field.y, q.y), .5f);
        const float w = __fadd_rn(__fadd_rn((float)m.field.z, q.z), .5f);
        const float value = tex3D<float>(sc.filter.linear, u, v, w);
        return sc.sdf_f16 ? value * m.lo.w : value;
    }
    uint32_t res = m.field.w;
    uint32_t cx = min(to_u32(floorf(q.x)), res - 2u);
    uint32_t cy = min(to_u32(floorf(q.y)), res - 2u);
    uint32_t cz = min(to_u32(floorf(q.z)), res - 2u);
    float fx = q.x - (float)cx, fy = q.y - (float)cy, fz = q.z - (float)cz;
    // One 32-byte (f32) or 16-byte (f16) corner record per cell instead of 8
    // texture fetches; the same texel values.
    float t[8];
    const uint32_t n = res - 1u;
    const uint32_t cell = __float_as_uint(m.hi.w) + (cz * n + cy) * n + cx;
    if (sc.sdf_f16) {
        const uint4 h = __ldg(static_cast<const uint4*>(sc.sdf_cells) + cell);
        const uint32_t w[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            t[2 * k] = __half2float(__ushort_as_half((unsigned short)(w[k] & 0xffffu)));
            t[2 * k + 1] = __half2float(__ushort_as_half((unsigned short)(w[k] >> 16)));
        }
    } else {
        const float4* c = static_cast<const float4*>(sc.sdf_cells) + 2 * (size_t)cell;
        const float4 a = __ldg(c), b = __ldg(c + 1);
        t[0] = a.x, t[1] = a.y, t[2] = a.z, t[3] = a.w;
        t[4] = b.x, t[5] = b.y, t[6] = b.z, t[7] = b.w;
    }
#if IRT_MARCH_FAST
    // The fast march: the same trilinear value as three lerp stages and the
    // f16 scale applied once — 14 operations for ~40; the rounding differs
    // from the weight sums in the last bits, as its approximate division and
    // square root do, far inside the field bound's voxel/128 margin.
    const float x0 = fmaf(fx, t[1] - t[0], t[0]), x1 = fmaf(fx, t[3] - t[2], t[2]);
    const float x2 = fmaf(fx, t[5] - t[4], t[4]), x3 = fmaf(fx, t[7] - t[6], t[6]);
    const float y0 = fmaf(fy, x1 - x0, x0), y1 = fmaf(fy, x3 - x2, x2);
    const float value = fmaf(fz, y1 - y0, y0);
    return sc.sdf_f16 ? value * m.lo.w : value;
#else
    if (sc.sdf_f16) {
        float s = m.lo.w;
#pragma unroll
        for (int k = 0; k < 8; k++) t[k] *= s;
    }
    float value = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float wx = (k & 1) ? fx : 1.f - fx;
        float wy = ((k >> 1) & 1) ? fy : 1.f - fy;
        float wz = (k >> 2) ? fz : 1.f - fz;
        value += t[k] * wx * wy * wz;
    }
    return value;
#endif
}

// sdf.wgsl:5-33
__device__ __forceinline__ float mesh_distance(const DevScene& sc, V3 p, const DMesh& m) {
    float geometry_bound = signed_box_distance(p, xyz(m.glo), xyz(m.ghi));
    if (m.glo.w > .5f) return geometry_bound;
    V3 lo = xyz(m.lo), hi = xyz(m.hi);
    V3 clamped = vmin(vmax(p, lo), hi);
    V3 q = (clamped - lo) * xyz(m.grid);
    float value = sample_field(sc, m, q);
    float bound = value - m.grid.w * (.5f + 1.f / 128.f);
    V3 outside = vmax(vmax(lo - p, p - hi), V3{0.f, 0.f, 0.f});
    float os = dot(outside, outside);
    if (os > 0.f) {
        float positive = wmax(bound, 0.f);
        bound = sqrtf(positive * positive + os);
    }
    if (bound > 0.f) bound *= m.ghi.w;
    float sphere_bound = length(p - xyz(m.sphere)) - m.sphere.w;
    return wmax(bound, wmax(geometry_bound, sphere_bound));
}

// sdf.wgsl:35-41 (returns the distance; the voxel is selected by the caller).
// rx/ry/rz are the rows of the object's inverse matrix.
__device__ __forceinline__ float object_distance_rows(const DevScene& sc, V3 p, float4 rx, float4 ry, float4 rz,
                                                      float scale, const DMesh& mesh) {
    V3 local = V3{rx.x * p.x + rx.y * p.y + rx.z * p.z + rx.w, ry.x * p.x + ry.y * p.y + ry.z * p.z + ry.w,
                  rz.x * p.x + rz.y * p.y + rz.z * p.z + rz.w};
    float d = mesh_distance(sc, local, mesh) * scale;
    if (d > 0.f) d *= .9999f;
    return d;
}
__device__ __forceinline__ float object_distance(const DevScene& sc, V3 p, const DObject& o) {
    DMesh mesh = load_mesh(sc.meshes, o.info.x);
    return object_distance_rows(sc, p, make_float4(o.c0.x, o.c1.x, o.c2.x, o.c3.x),
                                make_float4(o.c0.y, o.c1.y, o.c2.y, o.c3.y), make_float4(o.c0.z, o.c1.z, o.c2.z, o.c3.z),
                                __uint_as_float(o.info.z), mesh);
}

// Compact per-frame march scene (built on the host by irt_scene_update):
// preorder nodes then one record per object with its mesh folded in.
struct MNode {
    float4 a;  // lo.xyz, bits(escape index)
    float4 b;  // hi.xyz, bits(object id) for leaves, 0xffffffff otherwise
};
struct MObj {
    float4 rx, ry, rz;  // rows of the inverse model matrix
    float4 meta;        // bits(scale), bits(voxel diagonal * scale), mesh id, 0
    float4 lo, hi;      // mesh SDF bounds (lo.w: f16 texel scale)
    uint4 field;
    float4 grid, glo, ghi, sphere;
};
static_assert(sizeof(MNode) == 32, "MNode layout");
static_assert(sizeof(MObj) == 176, "MObj layout");

struct Dist {
    float best, voxel;
    uint32_t closest;
};

// sdf.wgsl:42-60 — the cursor only moves forward (escape links point past
// the subtree), so a walk visits at most 2N-1 nodes; a link that does not
// advance is reported through the error word and ends the walk.
__device__ __forceinline__ Dist scene_distance(const DevScene& sc, const irt_frame& f, V3 p, uint32_t hint,
                                               bool NeedSpacing) {
    Dist r{1e20f, f.sdf[1], hint};
    const uint32_t n = f.counts[3];
    if (hint < n) {
        DObject o = load_object(sc.objects, hint);
        r.best = object_distance(sc, p, o);
        if (NeedSpacing) r.voxel = __uint_as_float(o.info.w);
    }
    const uint32_t end = n * 2u - 1u;
    uint32_t cursor = 0;
    while (cursor < end) {
        DNode node = load_node(sc.nodes, cursor);
        V3 delta = vmax(vmax(xyz(node.lo) - p, p - xyz(node.hi)), V3{0.f, 0.f, 0.f});
        V3 lb = delta * .9998f;
        float b = wmax(r.best, 0.f);
        if (dot(lb, lb) > b * b) {
            uint32_t next = node.info.w;
            if (next <= cursor) {
                raise_error(sc.error, IRT_DEVERR_BVH_ESCAPE);
                break;
            }
            cursor = next;
            continue;
        }
        if (node.info.z == 1u) {
            uint32_t oid = node.info.x;
            if (oid != hint) {
                DObject o = load_object(sc.objects, oid);
                float d = object_distance(sc, p, o);
                if (d < r.best) {
                    r.best = d;
                    r.voxel = NeedSpacing ? __uint_as_float(o.info.w) : f.sdf[1];
                    r.closest = oid;
                }
            }
        }
        cursor++;
    }
    return r;
}

// The march of sdf.wgsl:61-81 split into steps shared by the per-pixel
// visibility() and the ray-queue march kernel, so both evaluate the same
// operations.  Each returns the resolved visibility, or -1 to continue.
struct MarchState {
    V3 origin, dir;
    float t, limit, result, previous;
    uint32_t closest, step;
};
// Top of march iteration `step`: budget first, then the ray length.
__device__ __forceinline__ float march_top(const MarchState& m, uint32_t max_steps) {
    if (m.step >= max_steps) return 0.f;  // a budget-exhausted ray is unresolved
    if (m.t >= m.limit) return wclamp(m.result, 0.f, 1.f);
    return -1.f;
}
__device__ __forceinline__ float march_begin(MarchState& m, V3 endpoint, float eps, uint32_t max_steps) {
    V3 delta = endpoint - m.origin;
    m.limit = length(delta) - eps;
    if (m.limit <= 0.f) return 1.f;
    m.dir = normalize(delta);
    m.t = eps;
    m.result = 1.f;
    m.previous = 1e20f;
    m.step = 0;
    return march_top(m, max_steps);
}
__device__ __forceinline__ V3 march_point(const MarchState& m) { return m.origin + m.dir * m.t; }
// Quilez improved penumbra update after a query of distance h.
__device__ __forceinline__ float march_after(MarchState& m, float h, float eps, float k, uint32_t max_steps) {
    if (h < eps) return 0.f;
    float y = h * h / (2.f * m.previous);
    float d = sqrtf(wmax(h * h - y * y, 0.f));
    if (m.t > y) m.result = wmin(m.result, k * d / (m.t - y));
    if (m.result < .001f) return 0.f;
    m.previous = h;
    m.t += h;
    m.step++;
    return march_top(m, max_steps);
}
__device__ __forceinline__ float clearance_epsilon(float eps, float voxel) { return wmax(eps, voxel * .65f); }

// sdf.wgsl:61-81 — soft-shadow visibility of `target` from surface point p.
__device__ __forceinline__ float visibility(const DevScene& sc, const irt_frame& f, V3 p, V3 n, V3 target,
                                            V3 end_normal) {
    const float eps = f.sdf[1];
    const uint32_t steps = to_u32(f.sdf[0]);
    MarchState m;
    Dist clearance = scene_distance(sc, f, p, 0xffffffffu, true);
    m.closest = clearance.closest;
    m.origin = p + n * clearance_epsilon(eps, clearance.voxel);
    V3 endpoint = target;
    if (dot(end_normal, end_normal) > .5f) {
        Dist e = scene_distance(sc, f, target, 0xffffffffu, true);
        endpoint = target + end_normal * clearance_epsilon(eps, e.voxel);
    }
    float r = march_begin(m, endpoint, eps, steps);
    while (r < 0.f) {
        Dist q = scene_distance(sc, f, march_point(m), m.closest, false);
        m.closest = q.closest;
        r = march_after(m, q.best, eps, f.sdf[2], steps);
    }
    return r;
}

}  // namespace irtd
