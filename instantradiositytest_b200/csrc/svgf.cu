// svgf.cu — svgf.wgsl (temporal moments, variance bootstrap, a-trous wavelet)
// as sm_100a CUDA.  One thread per pixel in 32x8 blocks; neighbour taps read
// the G-buffer guides and the radiance through L1 (2-D block locality).
#include <cuda_runtime.h>

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

template <class G>
struct Sv {
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
    __device__ __forceinline__ bool history_ok(int32_t px, int32_t py, int32_t qx, int32_t qy) const {
        if (f.flags[0] == 0u || f.flags[1] != f.size[3] || !inside(qx, qy)) return false;
        size_t q = idx(qx, qy);
        float d = __ldg(c.old_depth + q);
        if (d >= 1.f) return false;
        V3 a = position(px, py);
        V3 b = c.old_guide ? xyz(__ldg(c.old_guide + q)) : world(uvx(qx), uvy(qy), d, f.previous_inv_vp);
        return distance(a, b) < f.temporal[1] * wmax(distance(a, camera()), 1.f) &&
               dot(c.g.n(idx(px, py)), G::decode_normal(__ldg(c.old_normal + q))) > f.temporal[2];
    }
    // svgf.wgsl:28-31
    __device__ __forceinline__ Guide guide(int32_t x, int32_t y) const {
        Guide a;
        size_t i = idx(x, y);
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

// svgf.wgsl:45-76
template <class G, class R>
__global__ void __launch_bounds__(256) svgf_temporal_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                            const typename R::T* noisy, const typename R::T* old_radiance,
                                                            const float4* old_moments, typename R::T* radiance_out,
                                                            float4* moments_out) {
    int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    Sv<G> sv(f, c);
    if (x >= sv.W || y >= sv.H) return;
    size_t i = sv.idx(x, y);
    float4 c4 = R::load(noisy, i);
    V3 cc = V3{c4.x, c4.y, c4.z};
    float l = luminance(cc);
    V3 history = V3{0.f, 0.f, 0.f};
    float hm0 = 0.f, hm1 = 0.f, length_history = 0.f, total = 0.f;
    if (c.g.d(i) < 1.f) {
        float2 mv = c.g.mv(i);
        float px = (sv.uvx(x) - mv.x) * (float)sv.W - .5f;
        float py = (sv.uvy(y) - mv.y) * (float)sv.H - .5f;
        float flx = floorf(px), fly = floorf(py);
        int32_t bx = to_i32(flx), by = to_i32(fly);
        float fx = px - flx, fy = py - fly;
#pragma unroll
        for (int32_t yy = 0; yy < 2; yy++)
#pragma unroll
            for (int32_t xx = 0; xx < 2; xx++) {
                int32_t qx = bx + xx, qy = by + yy;
                if (!sv.history_ok(x, y, qx, qy)) continue;
                size_t q = sv.idx(qx, qy);
                float4 m = old_moments[q];
                if (m.z <= 0.f) continue;
                float wx = xx == 1 ? fx : 1.f - fx;
                float wy = yy == 1 ? fy : 1.f - fy;
                float w = wx * wy;
                float4 h = R::load(old_radiance, q);
                history = history + V3{h.x, h.y, h.z} * w;
                hm0 += m.x * w;
                hm1 += m.y * w;
                length_history += m.z * w;
                total += w;
            }
    }
    float age = 1.f;
    V3 result = cc;
    float m0 = l, m1 = l * l;
    if (total > .001f) {
        history = history / total;
        hm0 /= total;
        hm1 /= total;
        age = wmin(length_history / total + 1.f, f.temporal[3]);
        float lo = 1e20f, hi = 0.f;
        Guide a = sv.guide(x, y);
        for (int32_t yy = -1; yy <= 1; yy++)
            for (int32_t xx = -1; xx <= 1; xx++) {
                int32_t qx = min(max(x + xx, 0), sv.W - 1);
                int32_t qy = min(max(y + yy, 0), sv.H - 1);
                if (sv.geometry_weight(a, qx, qy, 1.f) > .01f) {
                    float4 n4 = R::load(noisy, sv.idx(qx, qy));
                    float v = luminance(V3{n4.x, n4.y, n4.z});
                    lo = wmin(lo, v);
                    hi = wmax(hi, v);
                }
            }
        float lh = luminance(history);
        history = history * (wclamp(lh, lo * .5f, hi * 1.5f + .001f) / wmax(lh, .000001f));
        float alpha = wmax(1.f - f.temporal[0], 1.f / age);
        result = V3{history.x * (1.f - alpha) + cc.x * alpha, history.y * (1.f - alpha) + cc.y * alpha,
                    history.z * (1.f - alpha) + cc.z * alpha};
        float beta = wmax(.2f, 1.f / age);
        float n0 = hm0 * (1.f - beta) + m0 * beta;
        float n1 = hm1 * (1.f - beta) + m1 * beta;
        m0 = n0;
        m1 = n1;
    }
    float variance = wmax(m1 - m0 * m0, 0.f);
    R::store(radiance_out, i, make_float4(result.x, result.y, result.z, wmin(sqrtf(variance), 65000.f)));
    moments_out[i] = make_float4(m0, m1, age, 0.f);
}

// svgf.wgsl:77-89
template <class G, class R>
__global__ void __launch_bounds__(256) svgf_variance_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                            const typename R::T* input, const float4* moments,
                                                            typename R::T* out) {
    int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    Sv<G> sv(f, c);
    if (x >= sv.W || y >= sv.H) return;
    size_t i = sv.idx(x, y);
    float4 in = R::load(input, i);
    float age = moments[i].z;
    float sigma = in.w;
    if (age < 4.f && c.g.d(i) < 1.f) {
        float s0 = 0.f, s1 = 0.f, total = 0.f;
        Guide a = sv.guide(x, y);
        for (int32_t yy = -3; yy <= 3; yy++)
            for (int32_t xx = -3; xx <= 3; xx++) {
                int32_t qx = x + xx, qy = y + yy;
                float w = sv.geometry_weight(a, qx, qy, 1.f);
                if (w <= 0.f) continue;
                float4 m = moments[sv.idx(qx, qy)];
                s0 += m.x * w;
                s1 += m.y * w;
                total += w;
            }
        float dn = wmax(total, .00001f);
        s0 /= dn;
        s1 /= dn;
        sigma = sqrtf(wmax(s1 - s0 * s0, 0.f) * 4.f / wmax(age, 1.f));
    }
    R::store(out, i, make_float4(in.x, in.y, in.z, wmin(sigma, 65000.f)));
}

// World position of every pixel, world(pixel_uv, depth, inv_vp)
// (common.wgsl:46-47) with its f32 operations rounded one by one, and in w
// the SVGF pixel scale distance(position, camera) / height (svgf.wgsl:30), or
// -1 where depth >= 1.  The lighting and SVGF kernels read positions from
// here instead of recomputing them per neighbour tap.
// With `previous` set, the same for the previous frame's depth and
// previous_inv_vp (the positions history_valid / history_ok compare with).
__global__ void __launch_bounds__(256) guide_kernel(const __grid_constant__ irt_frame f, const float* depth,
                                                    int previous, float4* out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t W = f.size[0];
    if (i >= (size_t)W * f.size[1]) return;
    uint32_t x = (uint32_t)(i % W), y = (uint32_t)(i / W);
    float d = __ldg(depth + i);
    V3 p = world(((float)x + .5f) / (float)W, ((float)y + .5f) / (float)f.size[1], d,
                 previous ? f.previous_inv_vp : f.inv_vp);
    float s = d < 1.f ? distance(p, V3{f.camera[0], f.camera[1], f.camera[2]}) / (float)f.size[1] : -1.f;
    out[i] = make_float4(p.x, p.y, p.z, s);
}

__device__ __forceinline__ float wavelet_kernel(int32_t x) {
    if (x == 0) return 1.f;
    if (x == 1 || x == -1) return 2.f / 3.f;
    return 1.f / 6.f;
}

// svgf.wgsl:91-110; `out2` (optional) receives a second copy of the result.
template <class G, class R>
__global__ void __launch_bounds__(256) svgf_atrous_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                          const typename R::T* input, typename R::T* out,
                                                          typename R::T* out2, int32_t step) {
    int32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t y = blockIdx.y * blockDim.y + threadIdx.y;
    Sv<G> sv(f, c);
    if (x >= sv.W || y >= sv.H) return;
    size_t i = sv.idx(x, y);
    float4 c4 = R::load(input, i);
    if (c.g.d(i) >= 1.f) {
        R::store(out, i, c4);
        if (out2) R::store(out2, i, c4);
        return;
    }
    float variance = 0.f, guide_weight = 0.f;
    Guide a = sv.guide(x, y);
#pragma unroll
    for (int32_t yy = -1; yy <= 1; yy++)
#pragma unroll
        for (int32_t xx = -1; xx <= 1; xx++) {
            int32_t qx = min(max(x + xx, 0), sv.W - 1);
            int32_t qy = min(max(y + yy, 0), sv.H - 1);
            float w = (xx == 0 ? 2.f : 1.f) * (yy == 0 ? 2.f : 1.f);
            float s = R::load(input, sv.idx(qx, qy)).w;
            variance += s * s * w;
            guide_weight += w;
        }
    float phi = 4.f * sqrtf(variance / wmax(guide_weight, .00001f)) + .0001f;
    V3 sum = V3{0.f, 0.f, 0.f};
    float total = 0.f, v = 0.f;
    float lc = luminance(V3{c4.x, c4.y, c4.z});
    for (int32_t yy = -2; yy <= 2; yy++)
        for (int32_t xx = -2; xx <= 2; xx++) {
            int32_t qx = x + xx * step, qy = y + yy * step;
            float geom = sv.geometry_weight(a, qx, qy, (float)step);
            if (geom <= 0.f) continue;
            float4 smp = R::load(input, sv.idx(qx, qy));
            float w = wavelet_kernel(xx) * wavelet_kernel(yy) * geom *
                      expf(-fabsf(luminance(V3{smp.x, smp.y, smp.z}) - lc) / phi);
            sum = sum + V3{smp.x, smp.y, smp.z} * w;
            v += smp.w * smp.w * w * w;
            total += w;
        }
    float dn = wmax(total, .00001f);
    float4 o = make_float4(sum.x / dn, sum.y / dn, sum.z / dn, wmin(sqrtf(v) / dn, 65000.f));
    R::store(out, i, o);
    if (out2) R::store(out2, i, o);
}

template <class G>
static SvgfCtx<G> make_ctx(const SvgfLaunch& L) {
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
    return c;
}

template <class G, class R>
static cudaError_t svgf_typed(const SvgfLaunch& L, int stage, cudaStream_t st) {
    SvgfCtx<G> c = make_ctx<G>(L);
    const irt_frame& f = *L.frame;
    typedef typename R::T T;
    dim3 block(32, 8);
    dim3 grid((f.size[0] + 31) / 32, (f.size[1] + 7) / 8);
    switch (stage) {
    case 0:
        svgf_temporal_kernel<G, R><<<grid, block, 0, st>>>(f, c, (const T*)L.in, (const T*)L.aux, (const float4*)L.moments_in,
                                                           (T*)L.out, (float4*)L.moments_out);
        break;
    case 1:
        svgf_variance_kernel<G, R><<<grid, block, 0, st>>>(f, c, (const T*)L.in, (const float4*)L.moments_in, (T*)L.out);
        break;
    case 2:
        svgf_atrous_kernel<G, R><<<grid, block, 0, st>>>(f, c, (const T*)L.in, (T*)L.out, (T*)L.out2, L.step);
        break;
    case 3:
    case 4: {
        size_t P = (size_t)f.size[0] * f.size[1];
        guide_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(f, stage == 3 ? L.gbuffer.depth : L.old_depth,
                                                                   stage == 4, (float4*)L.out);
    } break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace irtd

cudaError_t irt_launch_svgf(const SvgfLaunch& L, int stage, cudaStream_t st) {
    using namespace irtd;
    if (L.radiance_f16) {
        switch (L.gbuffer.format) {
        case IRT_GBUFFER_F32: return svgf_typed<GbF32, RadF16>(L, stage, st);
        case IRT_GBUFFER_F16: return svgf_typed<GbF16, RadF16>(L, stage, st);
        case IRT_GBUFFER_PACKED: return svgf_typed<GbPacked, RadF16>(L, stage, st);
        }
    } else {
        switch (L.gbuffer.format) {
        case IRT_GBUFFER_F32: return svgf_typed<GbF32, RadF32>(L, stage, st);
        case IRT_GBUFFER_F16: return svgf_typed<GbF16, RadF32>(L, stage, st);
        case IRT_GBUFFER_PACKED: return svgf_typed<GbPacked, RadF32>(L, stage, st);
        }
    }
    return cudaErrorInvalidValue;
}
