// lighting.cu — the 8 lighting entry points of lighting.wgsl as sm_100a CUDA.
//
// Two schedules over the same per-pixel device functions:
//   fused (default): reuse_kernel = candidates_direct + candidates_indirect +
//     temporal_direct + temporal_indirect (writes reservoirs [1]);
//     shade_kernel = spatial_direct + spatial_indirect + resolve_direct +
//     resolve_indirect (writes reservoirs [2], direct and combined radiance).
//   plain: one kernel per reference entry point (pass_kernel<Pass>).
// Both write bit-identical results: the fused kernels call the same device
// functions in the same order and keep intermediate reservoirs in registers
// (f32 values identical to their stored form).
// Threads: one per pixel, 32x8 blocks (warps span 32 consecutive pixels of a
// row, so every own-pixel access is a coalesced 128-bit vector access).
#include <cuda_runtime.h>

#include <type_traits>

#include "dev_sdf.cuh"
#include "kernels.h"

namespace irtd {

template <class G>
struct LightArgs {
    G g;
    DevScene sc;
    const irt_vpl* cur;
    const irt_vpl* prev;
    const irt_vpl* arch;
    const float* prev_depth;
    const typename G::NormalT* prev_normal;
    irt_reservoir* dres[3];
    irt_reservoir* ires[3];
    float4* direct_out;  // resolve_direct output (f32x4), may be null in fused mode
    void* noisy_out;     // resolve_indirect output (radiance format)
    RayRecord* rays;
    uint32_t* ray_counters;
    const float* vis;
    float4* pending;
    const float4* guide;      // world positions of this frame's pixels
    const float4* old_guide;  // ... of the previous frame's pixels
    const float4* feat;       // decoded (normal, rough), (colour, metal) per pixel, or null
};

// Scenes of at most kLightTable lights: the reuse pass evaluates every
// light's target (luminance of the unshadowed direct term) once per pixel,
// all independent, into a per-thread column of shared memory; the RIS loop
// and the temporal merge then read their light's entry.  Each entry is the
// same function of the same operands as the per-candidate evaluation, so
// the bits are too; what changes is that the 8 evaluations no longer wait
// on each other through the random stream.
constexpr uint32_t kLightTable = 8;
constexpr uint32_t kLightTableStride = 256;  // threads per block of the lighting kernels

template <class G>
struct Px {
    const irt_frame& f;
    const LightArgs<G>& a;
    uint32_t x, y;
    size_t id;
    const float* ltab = nullptr;  // light j's target at ltab[j * kLightTableStride], or null
    __device__ __forceinline__ Px(const irt_frame& fr, const LightArgs<G>& ar, uint32_t px, uint32_t py)
        : f(fr), a(ar), x(px), y(py), id((size_t)py * fr.size[0] + px) {}

    __device__ __forceinline__ V3 camera() const { return V3{f.camera[0], f.camera[1], f.camera[2]}; }
    __device__ __forceinline__ float uvx(uint32_t qx) const { return ((float)qx + .5f) / (float)f.size[0]; }
    __device__ __forceinline__ float uvy(uint32_t qy) const { return ((float)qy + .5f) / (float)f.size[1]; }
    __device__ __forceinline__ bool valid() const { return a.g.d(id) < 1.f; }
    // lighting.wgsl:30-34
    // world(pixel_uv(p), depth, inv_vp) of pixel i, precomputed per frame.
    __device__ __forceinline__ V3 position(size_t i) const { return xyz(__ldg(a.guide + i)); }
    // Normal of pixel i as the G-buffer stores it: for the f16 and packed
    // formats from the frame's decoded feature records (the same values the
    // decode gives), else from the f32 plane.
    __device__ __forceinline__ V3 normal_of(size_t i) const {
        if constexpr (!std::is_same<G, GbF32>::value)
            if (a.feat) return xyz(__ldg(a.feat + 2 * i));
        return a.g.n(i);
    }
    __device__ __forceinline__ Surface surface() const {
        Surface s;
        s.p = position(id);
        if constexpr (!std::is_same<G, GbF32>::value) {
            if (a.feat) {
                const float4 n = __ldg(a.feat + 2 * id), k = __ldg(a.feat + 2 * id + 1);
                s.n = normalize(xyz(n));
                s.color = xyz(k);
                s.rough = n.w;
                s.metal = k.w;
                surface_terms(s, camera());
                return s;
            }
        }
        s.n = normalize(a.g.n(id));
        s.color = a.g.c(id);
        float2 rm = a.g.pm(id);
        s.rough = rm.x;
        s.metal = rm.y;
        surface_terms(s, camera());
        return s;
    }
    // lighting.wgsl:36-40
    __device__ __forceinline__ bool compatible(const Surface& s, uint32_t qx, uint32_t qy) const {
        size_t q = (size_t)qy * f.size[0] + qx;
        float d = a.g.d(q);
        if (d >= 1.f) return false;
        V3 p = position(q);
        V3 n = normalize(normal_of(q));
        return dot(s.n, n) > f.temporal[2] && distance(s.p, p) < f.temporal[1] * wmax(distance(s.p, camera()), 1.f);
    }
    // lighting.wgsl:41-44
    __device__ __forceinline__ void reproject(int32_t& qx, int32_t& qy) const {
        float2 m = a.g.mv(id);
        float u = uvx(x) - m.x, v = uvy(y) - m.y;
        qx = to_i32(floorf(u * (float)f.size[0]));
        qy = to_i32(floorf(v * (float)f.size[1]));
    }
    // lighting.wgsl:45-50
    __device__ __forceinline__ bool history_valid(const Surface& s, int32_t qx, int32_t qy) const {
        if (f.flags[0] == 0u || f.flags[1] != f.size[3] || qx < 0 || qy < 0 || qx >= (int32_t)f.size[0] ||
            qy >= (int32_t)f.size[1])
            return false;
        size_t q = (size_t)qy * f.size[0] + (size_t)qx;
        if (!index_ok(a.sc.error, q, (size_t)f.size[0] * f.size[1])) return false;
        float d = __ldg(a.prev_depth + q);
        if (d >= 1.f) return false;
        // world((q + .5) / size, d, previous_inv_vp): the previous frame's
        // position of q, which is that frame's guide entry.
        V3 oldp = xyz(__ldg(a.old_guide + q));
        V3 pn = G::decode_normal(__ldg(a.prev_normal + q));
        return dot(s.n, pn) > f.temporal[2] && distance(s.p, oldp) < f.temporal[1] * wmax(distance(s.p, camera()), 1.f);
    }
    // lighting.wgsl:22-24
    __device__ __forceinline__ bool vpl_sample_valid(const Res& r) const {
        return r.generation == f.size[3] && r.target > 0.f && r.id < f.counts[1] &&
               f.size[2] - r.source <= to_u32(f.rr[2]);
    }
    // lighting.wgsl:25-29
    __device__ __forceinline__ DVpl selected_vpl(const Res& r) const {
        if (r.source == f.size[2]) return load_vpl(a.cur, r.id);
        if (r.source + 1u == f.size[2]) return load_vpl(a.prev, r.id);
        uint32_t slots = to_u32(f.rr[2]) + 1u;
        return load_vpl(a.arch, (size_t)(r.source % slots) * f.counts[1] + r.id);
    }
    // lighting.wgsl:86-89
    __device__ __forceinline__ void neighbor(uint32_t& rng, int32_t& qx, int32_t& qy) const {
        float angle = 2.f * kPI * rnd(rng);
        float radius = sqrtf(rnd(rng)) * (float)f.restir[3];
        qx = (int32_t)x + to_i32(rintf(cosf(angle) * radius));
        qy = (int32_t)y + to_i32(rintf(sinf(angle) * radius));
    }

    // ---------------------------------------------------------------- passes
    // lighting.wgsl:52-58
    __device__ __forceinline__ Res candidates_direct(bool ok, const Surface& s) const {
        Res r = res_empty(f);
        uint32_t rng = seed((uint32_t)id, 11u, f.size[2]);
        if (ok && f.counts[0] > 0u) {
            float pdf = 1.f / (float)f.counts[0];
            for (uint32_t i = 0; i < f.restir[0]; i++) {
                uint32_t lid = min(to_u32(rnd(rng) * (float)f.counts[0]), f.counts[0] - 1u);
                float target = ltab ? ltab[lid * kLightTableStride] : luminance(direct(s, load_light(a.sc.lights, lid)));
                res_add(r, lid, f.size[2], target, pdf, target / pdf, 1u, 0u, rng);
            }
        }
        return r;
    }
    // lighting.wgsl:59-65
    __device__ __forceinline__ Res candidates_indirect(bool ok, const Surface& s) const {
        Res r = res_empty(f);
        uint32_t rng = seed((uint32_t)id, 13u, f.size[2]);
        if (ok) {
            float pdf = 1.f / (float)f.counts[1];
            for (uint32_t i = 0; i < f.restir[1]; i++) {
                uint32_t vid = min(to_u32(rnd(rng) * (float)f.counts[1]), f.counts[1] - 1u);
                float target = luminance(indirect(s, load_vpl(a.cur, vid)));
                res_add(r, vid, f.size[2], target, pdf, target / pdf, 1u, 0u, rng);
            }
        }
        return r;
    }
    // lighting.wgsl:66-74 (hv = valid && history_valid)
    __device__ __forceinline__ void temporal_direct(Res& r, bool hv, const Surface& s, int32_t qx, int32_t qy) const {
        uint32_t rng = seed((uint32_t)id, 17u, f.size[2]);
        if (!hv) return;
        Res previous = cap(res_load(a.dres[2], (size_t)qy * f.size[0] + (size_t)qx), to_u32(f.rr[2]) * f.restir[0]);
        if (previous.generation == f.size[3] && previous.target > 0.f && previous.id < f.counts[0] &&
            previous.age < to_u32(f.rr[2])) {
            float target = ltab ? ltab[previous.id * kLightTableStride]
                                : luminance(direct(s, load_light(a.sc.lights, previous.id)));
            res_add(r, previous.id, previous.source, target, previous.pdf,
                    target * normalization(previous) * (float)previous.count, previous.count, previous.age + 1u, rng);
        }
    }
    // lighting.wgsl:75-85
    __device__ __forceinline__ void temporal_indirect(Res& r, bool hv, const Surface& s, int32_t qx, int32_t qy) const {
        uint32_t rng = seed((uint32_t)id, 19u, f.size[2]);
        if (!hv) return;
        Res previous = cap(res_load(a.ires[2], (size_t)qy * f.size[0] + (size_t)qx), to_u32(f.rr[2]) * f.restir[1]);
        if (vpl_sample_valid(previous)) {
            float target = luminance(indirect(s, selected_vpl(previous)));
            res_add(r, previous.id, previous.source, target, previous.pdf,
                    target * normalization(previous) * (float)previous.count, previous.count, previous.age + 1u, rng);
        }
    }
    // lighting.wgsl:90-97 / 98-105 — reservoir `r` is the pixel's own [1].
    template <int Dom>
    __device__ __forceinline__ Res spatial(Res r, bool ok, const Surface& s) const {
        uint32_t rng = seed((uint32_t)id, Dom == 0 ? 23u : 29u, f.size[2]);
        const irt_reservoir* in = Dom == 0 ? a.dres[1] : a.ires[1];
        if (ok) {
            for (uint32_t i = 0; i < f.restir[2]; i++) {
                int32_t qx, qy;
                neighbor(rng, qx, qy);
                if (qx < 0 || qy < 0 || qx >= (int32_t)f.size[0] || qy >= (int32_t)f.size[1]) continue;
                if (!index_ok(a.sc.error, (size_t)qy * f.size[0] + (size_t)qx, (size_t)f.size[0] * f.size[1]))
                    continue;
                if (!compatible(s, (uint32_t)qx, (uint32_t)qy)) continue;
                Res previous = res_load(in, (size_t)qy * f.size[0] + (size_t)qx);
                if (Dom == 0) {
                    if (previous.target > 0.f && index_ok(a.sc.error, previous.id, f.counts[0])) {
                        float target = luminance(direct(s, load_light(a.sc.lights, previous.id)));
                        res_add(r, previous.id, previous.source, target, previous.pdf,
                                target * normalization(previous) * (float)previous.count, previous.count, previous.age,
                                rng);
                    }
                } else if (vpl_sample_valid(previous)) {
                    float target = luminance(indirect(s, selected_vpl(previous)));
                    res_add(r, previous.id, previous.source, target, previous.pdf,
                            target * normalization(previous) * (float)previous.count, previous.count, previous.age, rng);
                }
            }
        }
        return cap(r, to_u32(f.rr[2]) * f.restir[Dom] * 8u);
    }
    // lighting.wgsl:106-122
    __device__ __forceinline__ V3 resolve_direct(bool ok, const Surface& s, const Res& d) const {
        V3 result = V3{0.f, 0.f, 0.f};
        if (ok) {
            uint32_t dbg = f.flags[2];
            if (d.target > 0.f && dbg != 2u && dbg < 3u && index_ok(a.sc.error, d.id, f.counts[0])) {
                DLight l = load_light(a.sc.lights, d.id);
                V3 value = direct(s, l);
                if (luminance(value) > 0.f) {
                    float vis = visibility(a.sc, f, s.p, s.n, xyz(l.ps), V3{0.f, 0.f, 0.f});
                    float k = normalization(d);
                    result = result + V3{value.x * k * vis, value.y * k * vis, value.z * k * vis};
                }
            }
            if (dbg == 3u) result = s.color;
            if (dbg == 4u) result = V3{s.n.x * .5f + .5f, s.n.y * .5f + .5f, s.n.z * .5f + .5f};
            if (dbg == 5u) {
                float2 m = a.g.mv(id);
                result = V3{wclamp(.5f + m.x * 50.f, 0.f, 1.f), wclamp(.5f + m.y * 50.f, 0.f, 1.f), .5f};
            }
        }
        return result;
    }
    // lighting.wgsl:123-134 (before the 65000 clamp)
    __device__ __forceinline__ V3 resolve_indirect(bool ok, const Surface& s, const Res& v, V3 result) const {
        uint32_t dbg = f.flags[2];
        if (ok && dbg != 1u && dbg < 3u) {
            if (vpl_sample_valid(v)) {
                DVpl smp = selected_vpl(v);
                V3 value = indirect(s, smp);
                if (luminance(value) > 0.f) {
                    float vis = visibility(a.sc, f, s.p, s.n, xyz(smp.pos), xyz(smp.nrm));
                    float k = normalization(v);
                    result = result + V3{value.x * k * vis, value.y * k * vis, value.z * k * vis};
                }
            }
        }
        return result;
    }
};

template <class R>
__device__ __forceinline__ void store_noisy(void* out, size_t i, V3 r) {
    R::store(reinterpret_cast<typename R::T*>(out), i, make_float4(wmin(r.x, 65000.f), wmin(r.y, 65000.f), wmin(r.z, 65000.f), 1.f));
}

// Per-frame prepared lights (normalised spot direction, cos of half angle).
__global__ void prepare_lights_kernel(const irt_light* lights, uint32_t n, irt_light* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DLight l = prepare_light(lights[i]);
    float4* o = reinterpret_cast<float4*>(out + i);
    o[0] = l.ps;
    o[1] = l.da;
    o[2] = l.ct;
}

// ---------------------------------------------------------------- fused kernels
template <class G>
__device__ __forceinline__ void reuse_body(const irt_frame& f, const LightArgs<G>& a, int keep_candidates, uint32_t x,
                                           uint32_t y) {
    if (x >= f.size[0] || y >= f.size[1]) return;
    Px<G> px(f, a, x, y);
    bool ok = px.valid();
    Surface s;
    if (ok) s = px.surface();
    __shared__ float ltab[kLightTable * kLightTableStride];
    const uint32_t t = threadIdx.y * blockDim.x + threadIdx.x;
    if (ok && f.counts[0] <= kLightTable && blockDim.x * blockDim.y == kLightTableStride) {
        const uint32_t n = f.counts[0];
#pragma unroll
        for (uint32_t j = 0; j < kLightTable; j++)
            if (j < n) ltab[j * kLightTableStride + t] = luminance(direct(s, load_light(a.sc.lights, j)));
        px.ltab = ltab + t;
    }
    Res rd = px.candidates_direct(ok, s);
    Res ri = px.candidates_indirect(ok, s);
    if (keep_candidates) {
        res_store(a.dres[0], px.id, rd);
        res_store(a.ires[0], px.id, ri);
    }
    int32_t qx, qy;
    px.reproject(qx, qy);
    bool hv = ok && px.history_valid(s, qx, qy);
    px.temporal_direct(rd, hv, s, qx, qy);
    px.temporal_indirect(ri, hv, s, qx, qy);
    res_store(a.dres[1], px.id, rd);
    res_store(a.ires[1], px.id, ri);
}

// Reuse and spatial-prep are latency bound (dependent PCG draws, reservoir
// and G-buffer gathers): 4 blocks of 256 per SM (64 registers, a few spilled
// values in L1) hide more of it than 3 blocks without spills (10 % and 2 %
// faster at 1920x1200).
template <class G>
__global__ void __launch_bounds__(256, 4) reuse_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ LightArgs<G> a,
                                                    int keep_candidates) {
    reuse_body<G>(f, a, keep_candidates, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

template <class G, class R>
__global__ void __launch_bounds__(256) shade_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ LightArgs<G> a) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= f.size[0] || y >= f.size[1]) return;
    Px<G> px(f, a, x, y);
    bool ok = px.valid();
    Surface s;
    if (ok) s = px.surface();
    Res rd = px.template spatial<0>(res_load(a.dres[1], px.id), ok, s);
    res_store(a.dres[2], px.id, rd);
    Res ri = px.template spatial<1>(res_load(a.ires[1], px.id), ok, s);
    res_store(a.ires[2], px.id, ri);
    V3 direct_result = px.resolve_direct(ok, s, rd);
    if (a.direct_out) a.direct_out[px.id] = make_float4(direct_result.x, direct_result.y, direct_result.z, 1.f);
    V3 total = px.resolve_indirect(ok, s, ri, direct_result);
    store_noisy<R>(a.noisy_out, px.id, total);
}

// ---------------------------------------------------------------- ray-queue resolve
// spatial_direct + spatial_indirect, then the resolve passes up to their
// visibility call: the pixel's contribution value * normalization is stored
// and, where the reference would march, a ray is appended to the queue
// (warp-aggregated: one atomic per ray class per warp).  Lanes of
// out-of-image pixels stay in the warp until the append so every ballot sees
// all 32 lanes.  VPL rays fill the queue from the front and light rays from
// the back (ray_slot), so the march takes whole runs of one class and
// neighbouring queue entries take the same phases (a VPL ray has one more
// clearance query); each ray's result slot is in its record, so the order
// changes no result.  The records' fields stay in registers (no indexed
// local array).
// Queue ends of the two ray classes: counter 0 fills from the front, 2 from the back.
constexpr uint32_t kVplCounter = 0, kLightCounter = 2;

template <class G, class R>
__device__ __forceinline__ void spatial_prep_body(const irt_frame& f, const LightArgs<G>& a, uint32_t x, uint32_t y) {
    const bool in = x < f.size[0] && y < f.size[1];
    bool ray_d = false, ray_i = false;
    V3 sp{0.f, 0.f, 0.f}, sn{0.f, 0.f, 0.f}, lpos{0.f, 0.f, 0.f}, vpos{0.f, 0.f, 0.f}, vnrm{0.f, 0.f, 0.f};
    size_t id = 0;
    if (in) {
        Px<G> px(f, a, x, y);
        id = px.id;
        bool ok = px.valid();
        Surface s;
        if (ok) s = px.surface();
        Res rd = px.template spatial<0>(res_load(a.dres[1], px.id), ok, s);
        res_store(a.dres[2], px.id, rd);
        Res ri = px.template spatial<1>(res_load(a.ires[1], px.id), ok, s);
        res_store(a.ires[2], px.id, ri);
        // resolve_direct (lighting.wgsl:106-122) up to visibility()
        float4 pd = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t dbg = f.flags[2];
        if (ok) {
            if (rd.target > 0.f && dbg != 2u && dbg < 3u && index_ok(a.sc.error, rd.id, f.counts[0])) {
                DLight l = load_light(a.sc.lights, rd.id);
                V3 value = direct(s, l);
                if (luminance(value) > 0.f) {
                    float k = normalization(rd);
                    pd = make_float4(value.x * k, value.y * k, value.z * k, 1.f);
                    ray_d = true;
                    lpos = xyz(l.ps);
                }
            }
            if (dbg == 3u) pd = make_float4(s.color.x, s.color.y, s.color.z, 0.f);
            if (dbg == 4u) pd = make_float4(s.n.x * .5f + .5f, s.n.y * .5f + .5f, s.n.z * .5f + .5f, 0.f);
            if (dbg == 5u) {
                float2 m = a.g.mv(px.id);
                pd = make_float4(wclamp(.5f + m.x * 50.f, 0.f, 1.f), wclamp(.5f + m.y * 50.f, 0.f, 1.f), .5f, 0.f);
            }
        }
        // resolve_indirect (lighting.wgsl:123-134) up to visibility()
        float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ok && dbg != 1u && dbg < 3u && px.vpl_sample_valid(ri)) {
            DVpl smp = px.selected_vpl(ri);
            V3 value = indirect(s, smp);
            if (luminance(value) > 0.f) {
                float k = normalization(ri);
                pi = make_float4(value.x * k, value.y * k, value.z * k, 1.f);
                ray_i = true;
                vpos = xyz(smp.pos);
                vnrm = xyz(smp.nrm);
            }
        }
        if (ray_d || ray_i) {
            sp = s.p;
            sn = s.n;
        }
        a.pending[id * 2] = pd;
        a.pending[id * 2 + 1] = pi;
    }
    // Warp-aggregated append.
    const unsigned full = 0xffffffffu;
    // lane within the warp for any 2-D block shape (warps take consecutive linear thread ids)
    const uint32_t lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31u;
    const unsigned bd = __ballot_sync(full, ray_d), bi = __ballot_sync(full, ray_i);
    const uint32_t nd = (uint32_t)__popc(bd), ni = (uint32_t)__popc(bi);
    // VPL rays from the front of the queue, light rays from the back
    // (ray_slot), so the march takes all VPL rays, then all light rays.
    uint32_t base_i = 0, base_d = 0;
    if (lane == 0) {
        if (ni) base_i = atomicAdd(a.ray_counters + kVplCounter, ni);
        if (nd) base_d = atomicAdd(a.ray_counters + kLightCounter, nd);
    }
    base_i = __shfl_sync(full, base_i, 0);
    base_d = __shfl_sync(full, base_d, 0);
    const uint32_t cap = 2u * f.size[0] * f.size[1];
    const unsigned below = (1u << lane) - 1u;
    if (ray_d) {
        const uint32_t k = base_d + (uint32_t)__popc(bd & below);
        float4* r = reinterpret_cast<float4*>(a.rays + (kLightCounter == 0 ? k : cap - 1u - k));
        r[0] = make_float4(sp.x, sp.y, sp.z, __uint_as_float((uint32_t)(id * 2)));
        r[1] = make_float4(sn.x, sn.y, sn.z, 0.f);
        r[2] = make_float4(lpos.x, lpos.y, lpos.z, 0.f);
        r[3] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (ray_i) {
        const uint32_t k = base_i + (uint32_t)__popc(bi & below);
        float4* r = reinterpret_cast<float4*>(a.rays + (kVplCounter == 0 ? k : cap - 1u - k));
        r[0] = make_float4(sp.x, sp.y, sp.z, __uint_as_float((uint32_t)(id * 2 + 1)));
        r[1] = make_float4(sn.x, sn.y, sn.z, 1.f);
        r[2] = make_float4(vpos.x, vpos.y, vpos.z, 0.f);
        r[3] = make_float4(vnrm.x, vnrm.y, vnrm.z, 0.f);
    }
}

template <class G, class R>
__global__ void __launch_bounds__(256, 4) spatial_prep_kernel(const __grid_constant__ irt_frame f,
                                                           const __grid_constant__ LightArgs<G> a) {
    spatial_prep_body<G, R>(f, a, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

// resolve_direct / resolve_indirect outputs from contribution x visibility:
// direct = c_d * vis_d (or the debug colour), noisy = min(direct + c_i * vis_i, 65000).
template <class R>
__device__ __forceinline__ void combine_body(const irt_frame& f, const float4* pending, const float* vis,
                                             float4* direct_out, void* noisy_out, size_t i) {
    size_t P = (size_t)f.size[0] * f.size[1];
    if (i >= P) return;
    float4 pd = pending[i * 2], pi = pending[i * 2 + 1];
    float2 v = reinterpret_cast<const float2*>(vis)[i];
    V3 result = V3{pd.x, pd.y, pd.z};
    if (pd.w != 0.f) result = V3{pd.x * v.x, pd.y * v.x, pd.z * v.x};
    direct_out[i] = make_float4(result.x, result.y, result.z, 1.f);
    if (pi.w != 0.f) result = result + V3{pi.x * v.y, pi.y * v.y, pi.z * v.y};
    store_noisy<R>(noisy_out, i, result);
}

template <class R>
__global__ void __launch_bounds__(256) combine_kernel(const __grid_constant__ irt_frame f, const float4* pending,
                                                      const float* vis, float4* direct_out, void* noisy_out) {
    combine_body<R>(f, pending, vis, direct_out, noisy_out, (size_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------- plain kernels
template <class G, class R, int Pass>
__global__ void __launch_bounds__(256) pass_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ LightArgs<G> a) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= f.size[0] || y >= f.size[1]) return;
    Px<G> px(f, a, x, y);
    bool ok = px.valid();
    Surface s;
    if (ok) s = px.surface();
    if (Pass == 0) {
        res_store(a.dres[0], px.id, px.candidates_direct(ok, s));
    } else if (Pass == 1) {
        res_store(a.ires[0], px.id, px.candidates_indirect(ok, s));
    } else if (Pass == 2 || Pass == 3) {
        int32_t qx, qy;
        px.reproject(qx, qy);
        bool hv = ok && px.history_valid(s, qx, qy);
        if (Pass == 2) {
            Res r = res_load(a.dres[0], px.id);
            px.temporal_direct(r, hv, s, qx, qy);
            res_store(a.dres[1], px.id, r);
        } else {
            Res r = res_load(a.ires[0], px.id);
            px.temporal_indirect(r, hv, s, qx, qy);
            res_store(a.ires[1], px.id, r);
        }
    } else if (Pass == 4) {
        res_store(a.dres[2], px.id, px.template spatial<0>(res_load(a.dres[1], px.id), ok, s));
    } else if (Pass == 5) {
        res_store(a.ires[2], px.id, px.template spatial<1>(res_load(a.ires[1], px.id), ok, s));
    } else if (Pass == 6) {
        V3 r = px.resolve_direct(ok, s, res_load(a.dres[2], px.id));
        a.direct_out[px.id] = make_float4(r.x, r.y, r.z, 1.f);
    } else {
        float4 d = a.direct_out[px.id];
        V3 total = px.resolve_indirect(ok, s, res_load(a.ires[2], px.id), V3{d.x, d.y, d.z});
        store_noisy<R>(a.noisy_out, px.id, total);
    }
}

// ---------------------------------------------------------------- batched views
// One launch covers every view of a batch: block b belongs to the view v
// with tile_start[v] <= b < tile_start[v + 1]; its tile within the view
// follows the view's width in blocks.  Frames and per-view arguments live
// in device tables; the per-pixel code is the single-view kernels'.
__device__ __forceinline__ uint32_t find_view(const uint32_t* __restrict__ start, uint32_t n, uint32_t b) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ void tile_xy(const irt_frame& f, uint32_t t, uint32_t& x, uint32_t& y) {
    uint32_t tiles_x = (f.size[0] + blockDim.x - 1) / blockDim.x;
    x = (t % tiles_x) * blockDim.x + threadIdx.x;
    y = (t / tiles_x) * blockDim.y + threadIdx.y;
}

// Copies a view's record into shared memory (4-byte words, every thread of
// the block), so the per-pixel code reads it like kernel parameters: from
// on-chip memory that no global store can alias.
template <class T>
__device__ __forceinline__ void stage_record(const T* __restrict__ src, T* dst) {
    static_assert(sizeof(T) % 4 == 0, "records are whole words");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (uint32_t i = tid; i < sizeof(T) / 4; i += nt) d[i] = __ldg(s + i);
}

template <class G>
__global__ void __launch_bounds__(256, 4) reuse_batched(const irt_frame* __restrict__ frames, const LightArgs<G>* __restrict__ args,
                                                     const uint32_t* __restrict__ tile_start, uint32_t n, int keep) {
    const uint32_t v = find_view(tile_start, n, blockIdx.x);
    __shared__ __align__(16) irt_frame f;
    __shared__ __align__(16) LightArgs<G> a;
    stage_record(frames + v, &f);
    stage_record(args + v, &a);
    __syncthreads();
    uint32_t x, y;
    tile_xy(f, blockIdx.x - __ldg(tile_start + v), x, y);
    reuse_body<G>(f, a, keep, x, y);
}

template <class G, class R>
__global__ void __launch_bounds__(256, 4) spatial_prep_batched(const irt_frame* __restrict__ frames,
                                                            const LightArgs<G>* __restrict__ args,
                                                            const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = find_view(tile_start, n, blockIdx.x);
    __shared__ __align__(16) irt_frame f;
    __shared__ __align__(16) LightArgs<G> a;
    stage_record(frames + v, &f);
    stage_record(args + v, &a);
    __syncthreads();
    uint32_t x, y;
    tile_xy(f, blockIdx.x - __ldg(tile_start + v), x, y);
    spatial_prep_body<G, R>(f, a, x, y);
}

template <class G, class R>
__global__ void __launch_bounds__(256) combine_batched(const irt_frame* __restrict__ frames,
                                                       const LightArgs<G>* __restrict__ args,
                                                       const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = find_view(tile_start, n, blockIdx.x);
    const LightArgs<G>& a = args[v];
    combine_body<R>(frames[v], a.pending, a.vis, a.direct_out, a.noisy_out,
                    (size_t)(blockIdx.x - __ldg(tile_start + v)) * blockDim.x + threadIdx.x);
}

// VPL archive slot frame % (H+1) of every view, and the ray-queue counters
// reset (src/renderer.rs:1873-1884).
template <class G>
__global__ void __launch_bounds__(256) archive_batched(const irt_frame* __restrict__ frames,
                                                       const LightArgs<G>* __restrict__ args, uint32_t n) {
    const uint32_t v = blockIdx.y;
    if (v >= n) return;
    const irt_frame& f = frames[v];
    const LightArgs<G>& a = args[v];
    const uint32_t count = f.counts[1];
    const uint32_t slots = to_u32(f.rr[2]) + 1u;
    const uint32_t slot = f.size[2] % slots;
    const float4* src = reinterpret_cast<const float4*>(a.cur);
    float4* dst = reinterpret_cast<float4*>(const_cast<irt_vpl*>(a.arch) + (size_t)slot * count);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count * 3u; i += gridDim.x * blockDim.x)
        dst[i] = src[i];
    if (blockIdx.x == 0 && threadIdx.x < 4) a.ray_counters[threadIdx.x] = 0u;
}

// ---------------------------------------------------------------- host launchers
template <class G>
static LightArgs<G> make_args(const LightingLaunch& L) {
    LightArgs<G> a;
    a.g.depth = L.gbuffer.depth;
    a.g.normal = reinterpret_cast<decltype(a.g.normal)>(L.gbuffer.normal);
    a.g.color = reinterpret_cast<decltype(a.g.color)>(L.gbuffer.color);
    a.g.params = reinterpret_cast<decltype(a.g.params)>(L.gbuffer.params);
    a.g.motion = reinterpret_cast<decltype(a.g.motion)>(L.gbuffer.motion);
    a.sc.objects = L.objects;
    a.sc.meshes = L.meshes;
    a.sc.nodes = L.nodes;
    a.sc.lights = L.lights;
    a.sc.atlas = L.atlas;
    a.sc.sdf_f16 = L.sdf_f16;
    a.sc.sdf_cells = L.sdf_cells;
    a.sc.filter = L.field_filter;
    a.sc.error = L.error;
    a.cur = L.cur_vpls;
    a.prev = L.prev_vpls;
    a.arch = L.archive;
    a.prev_depth = L.prev_depth;
    a.prev_normal = reinterpret_cast<const typename G::NormalT*>(L.prev_normal);
    for (int k = 0; k < 3; k++) {
        a.dres[k] = L.dres[k];
        a.ires[k] = L.ires[k];
    }
    a.direct_out = L.direct_out;
    a.noisy_out = L.noisy_out;
    a.rays = L.rays;
    a.ray_counters = L.ray_counters;
    a.vis = L.vis;
    a.pending = L.pending;
    a.guide = L.guide;
    a.old_guide = L.old_guide;
    a.feat = L.feat;
    return a;
}

template <class G, class R>
static cudaError_t launch_typed(const LightingLaunch& L, int stage, cudaStream_t st) {
    LightArgs<G> a = make_args<G>(L);
    const irt_frame& f = *L.frame;
    dim3 block(32, 8);
    dim3 grid((f.size[0] + 31) / 32, (f.size[1] + 7) / 8);
    switch (stage) {
    case kStageReuse: reuse_kernel<G><<<grid, block, 0, st>>>(f, a, L.keep_candidates); break;
    case kStageShade: shade_kernel<G, R><<<grid, block, 0, st>>>(f, a); break;
    case kStageSpatial: spatial_prep_kernel<G, R><<<grid, block, 0, st>>>(f, a); break;
    case kStageCombine: {
        size_t P = (size_t)f.size[0] * f.size[1];
        combine_kernel<R><<<(unsigned)((P + 255) / 256), 256, 0, st>>>(f, L.pending, L.vis, L.direct_out, L.noisy_out);
    } break;
    case 0: pass_kernel<G, R, 0><<<grid, block, 0, st>>>(f, a); break;
    case 1: pass_kernel<G, R, 1><<<grid, block, 0, st>>>(f, a); break;
    case 2: pass_kernel<G, R, 2><<<grid, block, 0, st>>>(f, a); break;
    case 3: pass_kernel<G, R, 3><<<grid, block, 0, st>>>(f, a); break;
    case 4: pass_kernel<G, R, 4><<<grid, block, 0, st>>>(f, a); break;
    case 5: pass_kernel<G, R, 5><<<grid, block, 0, st>>>(f, a); break;
    case 6: pass_kernel<G, R, 6><<<grid, block, 0, st>>>(f, a); break;
    case 7: pass_kernel<G, R, 7><<<grid, block, 0, st>>>(f, a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class G, class R>
static cudaError_t launch_batched_typed(const BatchLaunch& B, int stage, cudaStream_t st) {
    const irt_frame* frames = B.frames;
    const LightArgs<G>* args = static_cast<const LightArgs<G>*>(B.table);
    dim3 block(B.bx, B.by);
    switch (stage) {
    case kStageReuse: reuse_batched<G><<<B.tiles, block, 0, st>>>(frames, args, B.tile_start, B.n, B.keep); break;
    case kStageSpatial: spatial_prep_batched<G, R><<<B.tiles, block, 0, st>>>(frames, args, B.tile_start, B.n); break;
    case kStageCombine: combine_batched<G, R><<<B.tiles, 256, 0, st>>>(frames, args, B.tile_start, B.n); break;
    case kStageArchive: archive_batched<G><<<dim3(8, B.n), 256, 0, st>>>(frames, args, B.n); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace irtd

size_t irt_lighting_args_size(int gbuffer_format) {
    using namespace irtd;
    switch (gbuffer_format) {
    case IRT_GBUFFER_F32: return sizeof(LightArgs<GbF32>);
    case IRT_GBUFFER_F16: return sizeof(LightArgs<GbF16>);
    default: return sizeof(LightArgs<GbPacked>);
    }
}

void irt_lighting_args_fill(const LightingLaunch& L, void* out) {
    using namespace irtd;
    switch (L.gbuffer.format) {
    case IRT_GBUFFER_F32: *static_cast<LightArgs<GbF32>*>(out) = make_args<GbF32>(L); break;
    case IRT_GBUFFER_F16: *static_cast<LightArgs<GbF16>*>(out) = make_args<GbF16>(L); break;
    default: *static_cast<LightArgs<GbPacked>*>(out) = make_args<GbPacked>(L); break;
    }
}

cudaError_t irt_launch_lighting_batched(const BatchLaunch& B, int stage, cudaStream_t st) {
    using namespace irtd;
    if (B.n == 0) return cudaSuccess;
    if (B.radiance_f16) {
        switch (B.gbuffer_format) {
        case IRT_GBUFFER_F32: return launch_batched_typed<GbF32, RadF16>(B, stage, st);
        case IRT_GBUFFER_F16: return launch_batched_typed<GbF16, RadF16>(B, stage, st);
        case IRT_GBUFFER_PACKED: return launch_batched_typed<GbPacked, RadF16>(B, stage, st);
        }
    } else {
        switch (B.gbuffer_format) {
        case IRT_GBUFFER_F32: return launch_batched_typed<GbF32, RadF32>(B, stage, st);
        case IRT_GBUFFER_F16: return launch_batched_typed<GbF16, RadF32>(B, stage, st);
        case IRT_GBUFFER_PACKED: return launch_batched_typed<GbPacked, RadF32>(B, stage, st);
        }
    }
    return cudaErrorInvalidValue;
}

cudaError_t irt_launch_prepare_lights(const irt_light* lights, uint32_t n, irt_light* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    irtd::prepare_lights_kernel<<<(n + 127) / 128, 128, 0, st>>>(lights, n, out);
    return cudaGetLastError();
}

cudaError_t irt_launch_lighting(const LightingLaunch& L, int stage, cudaStream_t st) {
    using namespace irtd;
    if (L.radiance_f16) {
        switch (L.gbuffer.format) {
        case IRT_GBUFFER_F32: return launch_typed<GbF32, RadF16>(L, stage, st);
        case IRT_GBUFFER_F16: return launch_typed<GbF16, RadF16>(L, stage, st);
        case IRT_GBUFFER_PACKED: return launch_typed<GbPacked, RadF16>(L, stage, st);
        }
    } else {
        switch (L.gbuffer.format) {
        case IRT_GBUFFER_F32: return launch_typed<GbF32, RadF32>(L, stage, st);
        case IRT_GBUFFER_F16: return launch_typed<GbF16, RadF32>(L, stage, st);
        case IRT_GBUFFER_PACKED: return launch_typed<GbPacked, RadF32>(L, stage, st);
        }
    }
    return cudaErrorInvalidValue;
}
