// dev_svgf.cuh — shared helpers of the SVGF kernels (svgf.wgsl:18-44, :90):
// history test, per-pixel guides and the edge-stopping geometry weight.
#pragma once
#include <type_traits>

#include "dev_common.cuh"
#include "kernels.h"

namespace irtd {

template <class G>
struct SvgfCtx {
    G g;
    const float* old_depth;
    const typename G::NormalT* old_normal;
    // Per-pixel world positions of this frame and the previous one
    // (guide_kernel), or null to evaluate world() per tap; both give the
    // same values.
    const float4* guide;
    const float4* old_guide;
    // Per-pixel edge-stopping features of this frame (feature_kernel), two
    // float4 per pixel: (normal, roughness), (colour, metal) — the decoded
    // G-buffer values a tap reads, in 2 loads instead of 4 plane reads and
    // decodes; null to read the planes.  Requires `guide`.
    const float4* feat;
};

// x^64 as six squarings (the `pow(max(dot, 0), 64)` normal weight).
__device__ __forceinline__ float pow64(float x) {
    float y = x * x;
    y = y * y;
    y = y * y;
    y = y * y;
    y = y * y;
    return y * y;
}

struct Guide {
    V3 position, normal, color;
    float m0, m1, pixel_scale;
};

// Moment history storage.
//  MomF32: the reference's Rgba32Float (E[l], E[l^2], history length, 0).
//  MomF16: 8 bytes — mean and standard deviation of the luminance as two
//    halves, the history length as f32.  The second moment is kept central
//    (a deviation, not E[l^2]), so the f16 range holds it (luminance is
//    clamped at 65000; E[l^2] would overflow at 256) and the variance is
//    never formed as a difference of two rounded f16 values.  The kernels
//    accumulate and combine in f32 with the compensated forms below.
struct Moments {
    float mean, second, age;  // MomF32: second = E[l^2]; MomF16: second = deviation
};
struct MomF32 {
    typedef float4 T;
    static constexpr bool central = false;
    __device__ __forceinline__ static Moments load(const T* p, size_t i) {
        float4 m = p[i];
        return Moments{m.x, m.y, m.z};
    }
    __device__ __forceinline__ static void store(T* p, size_t i, Moments m) {
        p[i] = make_float4(m.mean, m.second, m.age, 0.f);
    }
};
struct MomF16 {
    typedef uint2 T;
    static constexpr bool central = true;
    __device__ __forceinline__ static Moments load(const T* p, size_t i) {
        uint2 m = p[i];
        __half2 h = *reinterpret_cast<const __half2*>(&m.x);
        return Moments{__low2float(h), __high2float(h), __uint_as_float(m.y)};
    }
    __device__ __forceinline__ static void store(T* p, size_t i, Moments m) {
        __half2 h = __floats2half2_rn(m.mean, m.second);
        p[i] = make_uint2(*reinterpret_cast<const uint32_t*>(&h), __float_as_uint(m.age));
    }
};

template <class G>
struct Sv {
    // Feature records are read for G-buffer formats that decode per tap.
    static constexpr bool kFeatures = !std::is_same<G, GbF32>::value;
    const irt_frame& f;
    const SvgfCtx<G>& c;
    int32_t W, H;
    __device__ __forceinline__ Sv(const irt_frame& fr, const SvgfCtx<G>& cx)
        : f(fr), c(cx), W((int32_t)fr.size[0]), H((int32_t)fr.size[1]) {}
    __device__ __forceinline__ size_t idx(int32_t x, int32_t y) const { return (size_t)y * (size_t)W + (size_t)x; }
    __device__ __forceinline__ bool inside(int32_t x, int32_t y) const { return x >= 0 && y >= 0 && x < W && y < H; }
    __device__ __forceinline__ V3 camera() const { return V3{f.camera[0], f.camera[1], f.camera[2]}; }
    __device__ __forceinline__ float uvx(int32_t x) const { return ((float)(uint32_t)x + .5f) / (float)W; }
    __device__ __forceinline__ float uvy(int32_t y) const { return ((float)(uint32_t)y + .5f) / (float)H; }
    // svgf.wgsl:19
    __device__ __forceinline__ V3 position(int32_t x, int32_t y) const {
        if (c.guide) return xyz(__ldg(c.guide + idx(x, y)));
        return world(uvx(x), uvy(y), c.g.d(idx(x, y)), f.inv_vp);
    }
    // svgf.wgsl:20-26
    // `a`, `n`: the pixel's position and (decoded) normal, `reach` =
    // temporal[1] * max(distance(a, camera), 1) — the same for its 4 taps.
    __device__ __forceinline__ bool history_ok(V3 a, V3 n, float reach, int32_t qx, int32_t qy) const {
        if (f.flags[0] == 0u || f.flags[1] != f.size[3] || !inside(qx, qy)) return false;
        size_t q = idx(qx, qy);
        float d = __ldg(c.old_depth + q);
        if (d >= 1.f) return false;
        V3 b = c.old_guide ? xyz(__ldg(c.old_guide + q)) : world(uvx(qx), uvy(qy), d, f.previous_inv_vp);
        return distance(a, b) < reach && dot(n, G::decode_normal(__ldg(c.old_normal + q))) > f.temporal[2];
    }
    __device__ __forceinline__ float history_reach(V3 a) const {
        return f.temporal[1] * wmax(distance(a, camera()), 1.f);
    }
    // svgf.wgsl:28-31
    __device__ __forceinline__ Guide guide(int32_t x, int32_t y) const {
        Guide a;
        size_t i = idx(x, y);
        if constexpr (kFeatures) {
            if (c.feat) {
                const float4 g = __ldg(c.guide + i), n = __ldg(c.feat + 2 * i), k = __ldg(c.feat + 2 * i + 1);
                a.position = xyz(g);
                a.normal = xyz(n);
                a.color = xyz(k);
                a.m0 = n.w;
                a.m1 = k.w;
                a.pixel_scale = g.w;  // distance(position, camera) / height (guide_kernel)
                return a;
            }
        }
        a.position = position(x, y);
        a.normal = c.g.n(i);
        a.color = c.g.c(i);
        float2 pm = c.g.pm(i);
        a.m0 = pm.x;
        a.m1 = pm.y;
        a.pixel_scale = distance(a.position, camera()) / (float)f.size[1];
        return a;
    }
    // svgf.wgsl:32-44
    __device__ __forceinline__ float geometry_weight(const Guide& a, int32_t qx, int32_t qy, float stride) const {
        if (!inside(qx, qy)) return 0.f;
        size_t q = idx(qx, qy);
        if constexpr (kFeatures) {
            if (c.feat) {
                const float4 g = __ldg(c.guide + q);
                if (g.w < 0.f) return 0.f;  // depth >= 1
                const float4 n = __ldg(c.feat + 2 * q), k = __ldg(c.feat + 2 * q + 1);
                float wn = pow64(wmax(dot(a.normal, xyz(n)), 0.f));
                float tolerance = wmax(.0001f, a.pixel_scale * stride * .5f);
                float wz = expf(-fabsf(dot(xyz(g) - a.position, a.normal)) / tolerance);
                V3 dc = a.color - xyz(k);
                float d0 = a.m0 - n.w, d1 = a.m1 - k.w;
                float wc = expf(-length(dc) * 8.f - sqrtf(d0 * d0 + d1 * d1) * 8.f);
                return wn * wz * wc;
            }
        }
        float dq = c.g.d(q);
        if (dq >= 1.f) return 0.f;
        V3 nq = c.g.n(q);
        float wn = pow64(wmax(dot(a.normal, nq), 0.f));
        V3 wq = c.guide ? xyz(__ldg(c.guide + q)) : world(uvx(qx), uvy(qy), dq, f.inv_vp);
        float tolerance = wmax(.0001f, a.pixel_scale * stride * .5f);
        float wz = expf(-fabsf(dot(wq - a.position, a.normal)) / tolerance);
        V3 dc = a.color - c.g.c(q);
        float2 pm = c.g.pm(q);
        float d0 = a.m0 - pm.x, d1 = a.m1 - pm.y;
        float wc = expf(-length(dc) * 8.f - sqrtf(d0 * d0 + d1 * d1) * 8.f);
        return wn * wz * wc;
    }
};

// Per-view record of a batched SVGF stage (the SvgfLaunch fields the stage
// reads, with the context in kernel form).
template <class G>
struct SView {
    SvgfCtx<G> c;
    const void* in;
    const void* aux;
    const void* moments_in;
    void* out;
    void* out2;
    void* moments_out;
    int32_t step;
};

__device__ __forceinline__ uint32_t svgf_find_view(const uint32_t* __restrict__ start, uint32_t n, uint32_t b) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}
// Copies a view's record into shared memory (4-byte words, every thread of
// the block), so the per-pixel code reads it like kernel parameters.
template <class T>
__device__ __forceinline__ void svgf_stage(const T* __restrict__ src, T* dst) {
    static_assert(sizeof(T) % 4 == 0, "records are whole words");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst);
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (uint32_t i = tid; i < sizeof(T) / 4; i += nt) d[i] = __ldg(s + i);
}
// Pixel of this thread in 2-D tile t of a view of width W.
__device__ __forceinline__ void svgf_tile_xy(uint32_t W, uint32_t t, int32_t& x, int32_t& y) {
    uint32_t tiles_x = (W + blockDim.x - 1) / blockDim.x;
    x = (int32_t)((t % tiles_x) * blockDim.x + threadIdx.x);
    y = (int32_t)((t / tiles_x) * blockDim.y + threadIdx.y);
}

// Calls fn(G{}, R{}, M{}) with the G-buffer, radiance and moment storage
// types a launch names.
template <class Fn>
__host__ inline cudaError_t dispatch_svgf(const SvgfLaunch& L, Fn&& fn) {
    auto with_m = [&](auto g, auto r) {
        return L.moments_f16 ? fn(g, r, MomF16{}) : fn(g, r, MomF32{});
    };
    auto with_r = [&](auto g) { return L.radiance_f16 ? with_m(g, RadF16{}) : with_m(g, RadF32{}); };
    switch (L.gbuffer.format) {
    case IRT_GBUFFER_F32: return with_r(GbF32{});
    case IRT_GBUFFER_F16: return with_r(GbF16{});
    case IRT_GBUFFER_PACKED: return with_r(GbPacked{});
    }
    return cudaErrorInvalidValue;
}

template <class G>
__host__ inline SvgfCtx<G> make_ctx(const SvgfLaunch& L) {
    SvgfCtx<G> c;
    c.g.depth = L.gbuffer.depth;
    c.g.normal = reinterpret_cast<decltype(c.g.normal)>(L.gbuffer.normal);
    c.g.color = reinterpret_cast<decltype(c.g.color)>(L.gbuffer.color);
    c.g.params = reinterpret_cast<decltype(c.g.params)>(L.gbuffer.params);
    c.g.motion = reinterpret_cast<decltype(c.g.motion)>(L.gbuffer.motion);
    c.old_depth = L.old_depth;
    c.old_normal = reinterpret_cast<const typename G::NormalT*>(L.old_normal);
    c.guide = L.guide;
    c.old_guide = L.old_guide;
    // Feature records pay off where a tap would decode (F16, packed); an F32
    // tap reads the planes as they are.
    c.feat = (L.guide && !std::is_same<G, GbF32>::value) ? L.feat : nullptr;
    return c;
}

}  // namespace irtd
