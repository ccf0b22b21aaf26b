// march.cu — persistent soft-shadow march over the ray queue.
//
// visibility() of sdf.wgsl:61-81 restated as a per-lane state machine over
// its scene_distance queries: the clearance query at the surface point, the
// endpoint clearance query for VPL rays, then up to sdf_max_steps march
// steps.  A lane that finishes its ray refills from its warp's reserved
// slice of the queue (one atomic per 32 entries, the records prefetched).
//
// scene_distance (sdf.wgsl:42-60) returns the minimum object distance: the
// walk skips a subtree only when its box bound exceeds the current best, and
// every object's distance is at least the distance to its BVH leaf box (the
// leaf box bounds the padded SDF box, which bounds the geometry box the
// distance is clamped to).  So visiting the same leaves in another order and
// skipping those whose box bound exceeds the current best yields the same
// best, the same closest object (ties aside) and the same voxel.  The march
// visits leaves in the order of a per-frame leaf-order cache: for the grid
// cell holding the query point, the leaves sorted by their box distance to
// the cell, stopping at the first whose bound exceeds the best so far.
// Points outside the grid, or past the cached entries, test every leaf.
// Per object the arithmetic is object_distance()'s, evaluated on records
// staged in shared memory.
//
// The loop is flattened to one object per lane and iteration (see Query):
// lanes at different stages of their queries evaluate objects together.
//
// This file is built twice: as is (IEEE division and square root, the
// arithmetic of the per-pixel visibility()), and through march_fast.cu with
// approximate division and square root for the default fast march.
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_sdf.cuh"
#include "kernels.h"

#ifndef IRT_MARCH_FAST
#define IRT_MARCH_FAST 0
#endif

namespace irtd {
#if IRT_MARCH_FAST
namespace fast {
#else
namespace exact {
#endif

enum : uint32_t { kClear = 0, kEndpoint = 1, kMarch = 2 };
// Resident warps: 64 registers a thread, no spills, 32 warps per SM.  In
// CTAs of 128 threads (the batched march): 9 CTAs at 56 registers spill and
// measured 3.82 ms, 7 CTAs 3.78 ms, 8 CTAs 3.56 ms per 1920x1200 frame.  The
// single-view march runs them as 4 CTAs of 256 threads, each staging the
// scene records once for 8 warps: 3.392 -> 3.371 ms against 8 CTAs of 128.
constexpr int kMarchBlocksPerSm = 8;
constexpr int kMarchThreads = 256;
constexpr int kMarchCtasPerSm = 4;
// Queue entries a warp reserves per atomic (one per lane): the queue counter
// then sees one atomic per ~30 warp iterations instead of about one per
// iteration (1920x1200 room: 3.51 -> 3.43 ms with the L2 prefetch of the
// reserved records, 3.46 without; 64 entries 3.45 ms).
constexpr uint32_t kRayChunk = 32;
constexpr uint32_t kNone = 0xffffffffu;

__device__ __forceinline__ float object_distance_rec(const DevScene& sc, V3 p, const MObj& o) {
    DMesh m;
    m.lo = o.lo;
    m.hi = o.hi;
    m.field = o.field;
    m.grid = o.grid;
    m.glo = o.glo;
    m.ghi = o.ghi;
    m.sphere = o.sphere;
    return object_distance_rows(sc, p, o.rx, o.ry, o.rz, o.meta.x, m);
}

struct Grid {
    const uint4* cells;
    float ox, oy, oz, ix, iy, iz;
};

// The march as one flattened loop: every iteration each lane evaluates at
// most one object, the next candidate of its current distance query — the
// hint object first (the previous closest, as scene_distance seeds it), then
// the leaf-order cache entries of the query point's cell that survive the
// walk's pruning tests (stopping at the first entry whose bound exceeds the
// best), then every leaf when the cached entries may not hold the minimum
// or the point is outside the grid.  A lane whose query has no candidate
// left completes it (the step of sdf.wgsl:61-81 it feeds), starts its ray's
// next query or takes a new ray, and finds that query's first candidate in
// the same iteration.  So the object evaluations of lanes at different
// stages of their queries (a hint, a second leaf, the first leaf of a new
// ray) issue together instead of in separate divergent sections; per query
// the candidates and their order are the same as a walk of one query at a
// time, so the results are too.
struct Query {
    V3 p;
    float best;
    uint32_t closest, hint;
    int32_t cur;          // next candidate: -1 hint, 0..7 cache entries, 8 after them, >= kAll all leaves
    const uint32_t* cw;   // the point's cache cell, or null outside the grid
};
constexpr int32_t kAfterEntries = (int32_t)kCellEntries;
constexpr int32_t kAll = 16;
constexpr int32_t kQueryDone = 0x7fffffff;

__device__ __forceinline__ void query_begin(Query& qy, const Grid& g, V3 p, uint32_t hint, uint32_t n) {
    qy.p = p;
    qy.best = 1e20f;
    qy.closest = hint;
    qy.hint = hint;
    const float fx = (p.x - g.ox) * g.ix, fy = (p.y - g.oy) * g.iy, fz = (p.z - g.oz) * g.iz;
    const float G = (float)kGridRes;
    const bool inside = fx >= 0.f && fy >= 0.f && fz >= 0.f && fx < G && fy < G && fz < G;
    qy.cw = nullptr;
    if (inside) {
        const uint32_t cell = ((uint32_t)fz * kGridRes + (uint32_t)fy) * kGridRes + (uint32_t)fx;
        qy.cw = reinterpret_cast<const uint32_t*>(g.cells + (size_t)cell * (kCellWords / 4));
    }
    qy.cur = hint < n ? -1 : (inside ? 0 : kAll);
}

// The walk's pruning test of leaf `oid`'s box against the best so far.
__device__ __forceinline__ bool leaf_may_hold_best(const MNode* nodes, const MObj* objs, V3 p, uint32_t oid,
                                                   float best) {
    const uint32_t leaf = __float_as_uint(objs[oid].meta.w);
    const float4 a = nodes[leaf].a, b = nodes[leaf].b;
    V3 delta = vmax(vmax(V3{a.x, a.y, a.z} - p, p - V3{b.x, b.y, b.z}), V3{0.f, 0.f, 0.f});
    V3 lb = delta * .9998f;
    float bb = wmax(best, 0.f);
    return !(dot(lb, lb) > bb * bb);
}

// Next object to evaluate for the query, or kNone when the query is complete.
__device__ __forceinline__ uint32_t query_next(Query& qy, const MNode* nodes, const MObj* objs, uint32_t n,
                                               uint32_t* err) {
    for (;;) {
        const int32_t c = qy.cur;
        if (c < 0) {  // the hint, unconditionally
            qy.cur = qy.cw ? 0 : kAll;
            return qy.hint;
        }
        if (c < kAfterEntries) {
            const uint32_t oid = (__ldg(qy.cw + (c >> 1)) >> ((c & 1) * 16)) & 0xffffu;
            if (__uint_as_float(__ldg(qy.cw + 4 + c)) > wmax(qy.best, 0.f) || oid == 0xffffu) {
                qy.cur = kQueryDone;
                return kNone;
            }
            qy.cur = c + 1;
            if (oid != qy.hint && index_ok(err, oid, n) && leaf_may_hold_best(nodes, objs, qy.p, oid, qy.best))
                return oid;
            continue;
        }
        if (c == kAfterEntries) {  // every cached entry fits: the ones left out may too
            qy.cur = __uint_as_float(__ldg(qy.cw + 12)) <= wmax(qy.best, 0.f) ? kAll : kQueryDone;
            continue;
        }
        if (c < kAll + (int32_t)n) {
            const uint32_t oid = (uint32_t)(c - kAll);
            qy.cur = c + 1;
            if (oid != qy.hint && leaf_may_hold_best(nodes, objs, qy.p, oid, qy.best)) return oid;
            continue;
        }
        return kNone;
    }
}

// Object `oid`'s distance folded into the query (the hint sets the best
// unconditionally, as scene_distance seeds it).
__device__ __forceinline__ void query_eval(Query& qy, const DevScene& sc, const MObj* objs, uint32_t oid) {
    const float d = object_distance_rec(sc, qy.p, objs[oid]);
    if (oid == qy.hint || d < qy.best) {
        qy.best = d;
        qy.closest = oid;
    }
}

// A completed query's step of visibility() (sdf.wgsl:61-81): after the
// clearance query the ray leaves the surface (and, for a VPL, queries the
// endpoint's clearance), after the endpoint query the march begins, after a
// march query the penumbra update.  Returns the visibility once the ray is
// resolved, else -1 with the ray's next query begun.
__device__ __forceinline__ float query_finish(Query& qy, MarchState& m, uint32_t& phase, const float4* rec,
                                              const Grid& grid, const MObj* objs, uint32_t n_obj, float eps, float k,
                                              uint32_t max_steps) {
    const float voxel = (phase != kMarch && qy.closest < n_obj) ? objs[qy.closest].meta.y : eps;
    float out = -1.f;
    if (phase == kClear) {
        m.closest = qy.closest;
        m.origin = m.origin + m.dir * clearance_epsilon(eps, voxel);
        const V3 endn = xyz(__ldg(rec + 3));
        if (dot(endn, endn) > .5f) {
            phase = kEndpoint;
        } else {
            phase = kMarch;
            out = march_begin(m, xyz(__ldg(rec + 2)), eps, max_steps);
        }
    } else if (phase == kEndpoint) {
        phase = kMarch;
        const V3 target = xyz(__ldg(rec + 2)), endn = xyz(__ldg(rec + 3));
        out = march_begin(m, target + endn * clearance_epsilon(eps, voxel), eps, max_steps);
    } else {
        m.closest = qy.closest;
        out = march_after(m, qy.best, eps, k, max_steps);
    }
    if (out < 0.f) {
        const V3 q = phase == kEndpoint ? xyz(__ldg(rec + 2)) : march_point(m);
        query_begin(qy, grid, q, phase == kMarch ? m.closest : kNone, n_obj);
    }
    return out;
}

// A warp's reserved slice [next, end) of a ray queue; `drained` once the
// queue counter has passed the queue's end.  Warp-uniform.
struct RaySlice {
    uint32_t next, end;
    bool drained;
};

// Queue indices for the warp's idle lanes (`need`, a ballot): this lane's
// index, or n_rays for none.  The slice is used first; a new reservation
// takes kRayChunk entries while more than `keep` entries are left (two
// chunks per warp of the grid: the warp's own slice end trails the counter
// by up to one), else what the idle lanes still need.  The lanes prefetch a
// new chunk's records into L2, so the loads of the lanes that take them
// later hit L2 instead of DRAM.
__device__ __forceinline__ uint32_t slice_take(RaySlice& s, unsigned need, uint32_t* counter, uint32_t n_rays,
                                               uint32_t keep, int lane, const RayRecord* rays, uint32_t front,
                                               uint32_t cap) {
    const unsigned full = 0xffffffffu;
    const uint32_t cnt = (uint32_t)__popc(need);
    const uint32_t avail = s.end - s.next;
    const uint32_t rank = (uint32_t)__popc(need & ((1u << lane) - 1u));
    uint32_t idx = rank < avail ? s.next + rank : n_rays;
    if (avail >= cnt) {
        s.next += cnt;
    } else if (s.drained) {
        s.next = s.end;
    } else {
        const uint32_t want = s.end + keep < n_rays ? kRayChunk : cnt - avail;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(counter, want);
        base = __shfl_sync(full, base, 0);
        if (rank >= avail) idx = base + (rank - avail);
        if (base >= n_rays) {
            s.drained = true;
            s.next = s.end = 0;
        } else {
            if ((uint32_t)lane < want && base + (uint32_t)lane < n_rays) {
                const uint32_t slot = ray_slot(base + (uint32_t)lane, front, cap);
                if (slot < cap) asm volatile("prefetch.global.L2 [%0];" ::"l"(rays + slot));
            }
            s.drained = base + want >= n_rays;
            s.end = s.drained ? n_rays : base + want;
            s.next = min(base + (cnt - avail), s.end);
        }
    }
    return idx;
}

__device__ __forceinline__ void march_reset(MarchState& m) {
    m.closest = kNone;
    m.origin = V3{0.f, 0.f, 0.f};
    m.dir = V3{0.f, 0.f, 0.f};
    m.t = m.limit = 0.f;
    m.result = 1.f;
    m.previous = 1e20f;
    m.step = 0;
}

__global__ void __launch_bounds__(kMarchThreads, kMarchCtasPerSm) march_kernel(const __grid_constant__ irt_frame f, const DevScene sc,
                                                    const float4* __restrict__ march_scene, uint32_t scene_vec4,
                                                    const Grid grid, const RayRecord* __restrict__ rays,
                                                    uint32_t* counters, float* __restrict__ vis) {
    extern __shared__ float4 smem[];
    for (uint32_t i = threadIdx.x; i < scene_vec4; i += blockDim.x) smem[i] = __ldg(march_scene + i);
    __syncthreads();
    const uint32_t n_obj = f.counts[3];
    const MNode* nodes = reinterpret_cast<const MNode*>(smem);
    const MObj* objs = reinterpret_cast<const MObj*>(smem + 2 * (2 * n_obj - 1));

    const uint32_t front = *(volatile uint32_t*)&counters[0];
    const uint32_t n_rays = front + *(volatile uint32_t*)&counters[2];
    const uint32_t cap = 2u * f.size[0] * f.size[1];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const float eps = f.sdf[1];
    const uint32_t max_steps = to_u32(f.sdf[0]);

    bool active = false;
    bool exhausted = false;  // warp-uniform: the queue has no rays left
    // A lane keeps its ray's index and re-reads the record's target, endpoint
    // normal and output slot where a step needs them (L1/L2 hits), which
    // keeps fewer values live across the loop.
    uint32_t phase = kClear, ridx = 0;
    MarchState m;
    march_reset(m);
    Query qy;
    qy.cur = kQueryDone;
    RaySlice slice{0u, 0u, false};
    const uint32_t keep = 2u * gridDim.x * (blockDim.x / 32u) * kRayChunk;
    for (;;) {
        if (!exhausted) {
            const unsigned need = __ballot_sync(full, !active);
            if (need) {
                const uint32_t idx = slice_take(slice, need, &counters[1], n_rays, keep, lane, rays, front, cap);
                exhausted = slice.drained && slice.next >= slice.end;
                if (!active) {
                    if (idx < n_rays && index_ok(sc.error, ray_slot(idx, front, cap), cap)) {
                        ridx = ray_slot(idx, front, cap);
                        const float4* r = reinterpret_cast<const float4*>(rays + ridx);
                        float4 a = __ldg(r), b = __ldg(r + 1);
                        m.origin = V3{a.x, a.y, a.z};  // surface point until the clearance query
                        m.dir = V3{b.x, b.y, b.z};     // surface normal until the march begins
                        phase = kClear;
                        active = true;
                        query_begin(qy, grid, m.origin, kNone, n_obj);
                    }
                }
            }
        }
        if (!__any_sync(full, active)) break;
        if (!active) continue;

        uint32_t oid = query_next(qy, nodes, objs, n_obj, sc.error);
        while (oid == kNone) {
            const float4* rec = reinterpret_cast<const float4*>(rays + ridx);
            const float out = query_finish(qy, m, phase, rec, grid, objs, n_obj, eps, f.sdf[2], max_steps);
            if (out >= 0.f) {
                const uint32_t slot = __float_as_uint(__ldg(rec).w);
                if (index_ok(sc.error, slot, cap)) vis[slot] = out;
                active = false;
                break;
            }
            oid = query_next(qy, nodes, objs, n_obj, sc.error);
        }
        if (oid != kNone) query_eval(qy, sc, objs, oid);
    }
}

// Batched march: for each scene group the CTA stages the group record and
// its compact scene in shared memory, then its warps consume the group's ray
// queues (one per view) in order with the same flattened loop; a lane keeps
// the address of its ray record and the index of the queue it came from.
constexpr uint32_t kGroupVec4 = (uint32_t)((sizeof(MarchGroup) + 15) / 16);

__global__ void __launch_bounds__(128, kMarchBlocksPerSm) march_batched_kernel(const MarchGroup* __restrict__ groups, uint32_t n_groups,
                                                            const MarchQueue* __restrict__ queues) {
    extern __shared__ float4 smem[];
    const MarchGroup& G = *reinterpret_cast<const MarchGroup*>(smem);
    float4* scene_smem = smem + kGroupVec4;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    for (uint32_t g = 0; g < n_groups; g++) {
        __syncthreads();  // every warp is done with the previous group's records
        const float4* gsrc = reinterpret_cast<const float4*>(groups + g);
        for (uint32_t i = threadIdx.x; i < kGroupVec4; i += blockDim.x) smem[i] = __ldg(gsrc + i);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < G.scene_vec4; i += blockDim.x) scene_smem[i] = __ldg(G.march_scene + i);
        __syncthreads();
        const irt_frame& f = G.f;
        DevScene sc;
        sc.objects = G.objects;
        sc.meshes = G.meshes;
        sc.nodes = G.nodes;
        sc.lights = nullptr;
        sc.atlas = G.atlas;
        sc.sdf_f16 = G.sdf_f16;
        sc.sdf_cells = G.sdf_cells;
        sc.filter = G.field_filter;
        sc.error = G.error;
        Grid grid;
        grid.cells = G.cells;
        grid.ox = G.grid_org[0];
        grid.oy = G.grid_org[1];
        grid.oz = G.grid_org[2];
        grid.ix = G.grid_inv[0];
        grid.iy = G.grid_inv[1];
        grid.iz = G.grid_inv[2];
        const uint32_t n_obj = f.counts[3];
        const MNode* nodes = reinterpret_cast<const MNode*>(scene_smem);
        const MObj* objs = reinterpret_cast<const MObj*>(scene_smem + 2 * (2 * n_obj - 1));
        const float eps = f.sdf[1];
        const uint32_t max_steps = to_u32(f.sdf[0]);

        uint32_t q = G.q_begin;
        bool exhausted = q >= G.q_end;
        uint32_t front = exhausted ? 0u : *(volatile const uint32_t*)&queues[q].counters[0];
        uint32_t n_rays = exhausted ? 0u : front + *(volatile const uint32_t*)&queues[q].counters[2];
        bool active = false;
        uint32_t phase = kClear, lq = 0;
        const float4* rec = nullptr;
        MarchState m;
        march_reset(m);
        Query qy;
        qy.cur = kQueryDone;
        RaySlice slice{0u, 0u, false};
        const uint32_t keep = 2u * gridDim.x * (blockDim.x / 32u) * kRayChunk;
        for (;;) {
            if (!exhausted) {
                const unsigned need = __ballot_sync(full, !active);
                if (need) {
                    const MarchQueue& Q = queues[q];
                    const uint32_t idx = slice_take(slice, need, &Q.counters[1], n_rays, keep, lane, Q.rays, front,
                                                    Q.cap);
                    if (!active) {
                        if (idx < n_rays && index_ok(sc.error, ray_slot(idx, front, Q.cap), Q.cap)) {
                            rec = reinterpret_cast<const float4*>(Q.rays + ray_slot(idx, front, Q.cap));
                            float4 a = __ldg(rec), b = __ldg(rec + 1);
                            m.origin = V3{a.x, a.y, a.z};
                            m.dir = V3{b.x, b.y, b.z};
                            phase = kClear;
                            lq = q;
                            active = true;
                            query_begin(qy, grid, m.origin, kNone, n_obj);
                        }
                    }
                    if (slice.drained && slice.next >= slice.end) {  // this queue is used up: the next view's
                        slice = RaySlice{0u, 0u, false};
                        q++;
                        if (q >= G.q_end) exhausted = true;
                        else {
                            front = *(volatile const uint32_t*)&queues[q].counters[0];
                            n_rays = front + *(volatile const uint32_t*)&queues[q].counters[2];
                        }
                    }
                }
            }
            if (!__any_sync(full, active)) {
                if (exhausted) break;
                continue;
            }
            if (!active) continue;

            uint32_t oid = query_next(qy, nodes, objs, n_obj, sc.error);
            while (oid == kNone) {
                const float out = query_finish(qy, m, phase, rec, grid, objs, n_obj, eps, f.sdf[2], max_steps);
                if (out >= 0.f) {
                    float* vis = queues[lq].vis;
                    const uint32_t slot = __float_as_uint(__ldg(rec).w);
                    if (index_ok(sc.error, slot, queues[lq].cap)) vis[slot] = out;
                    active = false;
                    break;
                }
                oid = query_next(qy, nodes, objs, n_obj, sc.error);
            }
            if (oid != kNone) query_eval(qy, sc, objs, oid);
        }
    }
}

}  // namespace fast / exact
}  // namespace irtd

#if IRT_MARCH_FAST
#define IRT_MARCH_NS irtd::fast
#define IRT_MARCH_LAUNCH irt_launch_march_fast
#else
#define IRT_MARCH_NS irtd::exact
#define IRT_MARCH_LAUNCH irt_launch_march_exact
#endif

// The carveout (percent of the SM's shared-memory maximum) that holds
// `blocks` CTAs of `smem` dynamic bytes plus the runtime's per-CTA reserve,
// and no more: the rest of the unified storage stays L1, where the leaf-order
// cache cells and SDF corner records of the march hit (1920x1200 room:
// 3.555 -> 3.531 ms against the driver's own choice; 50 % measured 3.589).
static cudaError_t march_prefer_l1(const void* kernel, uint32_t smem, int blocks) {
    int device = 0, per_sm = 0, reserved = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) return cudaSuccess;
    const long long need = (long long)blocks * ((long long)smem + reserved);
    const int pct = (int)std::min(100LL, (need * 100 + per_sm - 1) / per_sm);
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

cudaError_t IRT_MARCH_LAUNCH(const MarchLaunch& M, cudaStream_t st) {
    using namespace irtd;
    using namespace IRT_MARCH_NS;
    const uint32_t smem = irt_march_scene_bytes(M.frame->counts[3]);
    thread_local int configured_device = -1;
    thread_local uint32_t configured_smem = 0;
    thread_local int blocks_per_sm = 0;
    int device = 0;
    cudaGetDevice(&device);
    if (smem != configured_smem || device != configured_device) {
        configured_device = device;
        cudaError_t e = cudaFuncSetAttribute(march_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = march_prefer_l1((const void*)march_kernel, smem, kMarchCtasPerSm);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, march_kernel, kMarchThreads, smem);
        if (e != cudaSuccess) return e;
        if (blocks_per_sm < 1) return cudaErrorInvalidConfiguration;
        configured_smem = smem;
    }
    DevScene sc;
    sc.objects = M.objects;
    sc.meshes = M.meshes;
    sc.nodes = M.nodes;
    sc.lights = nullptr;
    sc.atlas = M.atlas;
    sc.sdf_f16 = M.sdf_f16;
    sc.sdf_cells = M.sdf_cells;
    sc.filter = M.field_filter;
    sc.error = M.error;
    Grid g;
    g.cells = M.cells;
    g.ox = M.grid_org[0];
    g.oy = M.grid_org[1];
    g.oz = M.grid_org[2];
    g.ix = M.grid_inv[0];
    g.iy = M.grid_inv[1];
    g.iz = M.grid_inv[2];
    march_kernel<<<M.num_sms * blocks_per_sm, kMarchThreads, smem, st>>>(*M.frame, sc, M.march_scene, smem / 16, g, M.rays,
                                                                M.ray_counters, M.vis);
    return cudaGetLastError();
}

#if IRT_MARCH_FAST
#define IRT_MARCH_BATCHED_LAUNCH irt_launch_march_batched_fast
#else
#define IRT_MARCH_BATCHED_LAUNCH irt_launch_march_batched_exact
#endif

cudaError_t IRT_MARCH_BATCHED_LAUNCH(const MarchBatch& M, cudaStream_t st) {
    using namespace irtd;
    using namespace IRT_MARCH_NS;
    if (M.n_groups == 0) return cudaSuccess;
    const uint32_t smem = kGroupVec4 * 16 + M.max_scene_bytes;
    thread_local int configured_device = -1;
    thread_local uint32_t configured_smem = 0;
    thread_local int max_blocks = 0;
    int device = 0;
    cudaGetDevice(&device);
    if (smem != configured_smem || device != configured_device) {
        configured_device = device;
        cudaError_t e = cudaFuncSetAttribute(march_batched_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = march_prefer_l1((const void*)march_batched_kernel, smem, kMarchBlocksPerSm);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&max_blocks, march_batched_kernel, 128, smem);
        if (e != cudaSuccess) return e;
        if (max_blocks < 1) return cudaErrorInvalidConfiguration;
        configured_smem = smem;
    }
    const int bps = M.blocks_per_sm > 0 && M.blocks_per_sm < max_blocks ? M.blocks_per_sm : max_blocks;
    march_batched_kernel<<<M.num_sms * bps, 128, smem, st>>>(M.groups, M.n_groups, M.queues);
    return cudaGetLastError();
}

#if !IRT_MARCH_FAST
cudaError_t irt_launch_march_batched_fast(const MarchBatch& M, cudaStream_t st);

cudaError_t irt_launch_march_batched(const MarchBatch& M, cudaStream_t st) {
    return M.fast ? irt_launch_march_batched_fast(M, st) : irt_launch_march_batched_exact(M, st);
}

uint32_t irt_march_scene_bytes(uint32_t object_count) {
    return (2 * object_count - 1) * (uint32_t)sizeof(irtd::MNode) + object_count * (uint32_t)sizeof(irtd::MObj);
}

cudaError_t irt_launch_march_fast(const MarchLaunch& M, cudaStream_t st);

cudaError_t irt_launch_march(const MarchLaunch& M, cudaStream_t st) {
    return M.fast ? irt_launch_march_fast(M, st) : irt_launch_march_exact(M, st);
}
#endif
