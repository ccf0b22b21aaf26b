// svgf_spatial.cu — svgf_variance (svgf.wgsl:77-89) and svgf_atrous
// (svgf.wgsl:90-110) as sm_100a CUDA, built with fast math (approximate
// exp, division and square root): these passes only weight and average
// radiance, and their inputs (positions, history length) come exactly from
// the guide and temporal kernels.  One thread per pixel (variance in 32x8
// blocks, a-trous in blocks of 256 pixels of a row); neighbour taps read
// through L1.
#include <cuda_runtime.h>

#include "dev_svgf.cuh"
#include "kernels.h"

namespace irtd {

// svgf.wgsl:77-89
// With MomF16 (mean, deviation) moments the 7x7 sums are taken about the
// centre pixel's mean (shifted data), so E[l^2] - E[l]^2 is formed from
// small numbers: s0 = sum w (m - K), s1 = sum w (dev^2 + (m - K)^2).
template <class G, class R, class M>
__device__ __forceinline__ void variance_body(const irt_frame& f, const SvgfCtx<G>& c, const typename R::T* input,
                                              const typename M::T* moments, typename R::T* out, int32_t x, int32_t y) {
    Sv<G> sv(f, c);
    if (x >= sv.W || y >= sv.H) return;
    size_t i = sv.idx(x, y);
    float4 in = R::load(input, i);
    Moments centre = M::load(moments, i);
    float age = centre.age;
    float sigma = in.w;
    if (age < 4.f && c.g.d(i) < 1.f) {
        float s0 = 0.f, s1 = 0.f, total = 0.f;
        const float K = M::central ? centre.mean : 0.f;
        Guide a = sv.guide(x, y);
        for (int32_t yy = -3; yy <= 3; yy++)
            for (int32_t xx = -3; xx <= 3; xx++) {
                int32_t qx = x + xx, qy = y + yy;
                float w = sv.geometry_weight(a, qx, qy, 1.f);
                if (w <= 0.f) continue;
                Moments m = M::load(moments, sv.idx(qx, qy));
                if constexpr (M::central) {
                    float d = m.mean - K;
                    s0 += d * w;
                    s1 += (m.second * m.second + d * d) * w;
                } else {
                    s0 += m.mean * w;
                    s1 += m.second * w;
                }
                total += w;
            }
        float dn = wmax(total, .00001f);
        s0 /= dn;
        s1 /= dn;
        sigma = sqrtf(wmax(s1 - s0 * s0, 0.f) * 4.f / wmax(age, 1.f));
    }
    R::store(out, i, make_float4(in.x, in.y, in.z, wmin(sigma, 65000.f)));
}

template <class G, class R, class M>
__global__ void __launch_bounds__(256) svgf_variance_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                            const typename R::T* input, const typename M::T* moments,
                                                            typename R::T* out) {
    variance_body<G, R, M>(f, c, input, moments, out, blockIdx.x * blockDim.x + threadIdx.x,
                           blockIdx.y * blockDim.y + threadIdx.y);
}

__device__ __forceinline__ float wavelet_kernel(int32_t x) {
    if (x == 0) return 1.f;
    if (x == 1 || x == -1) return 2.f / 3.f;
    return 1.f / 6.f;
}

// svgf.wgsl:91-110; `out2` (optional) receives a second copy of the result.
template <class G, class R>
__device__ __forceinline__ void atrous_body(const irt_frame& f, const SvgfCtx<G>& c, const typename R::T* input,
                                            typename R::T* out, typename R::T* out2, int32_t step, int32_t x,
                                            int32_t y) {
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
    auto tap = [&](int32_t xx, int32_t yy) {
        int32_t qx = x + xx * step, qy = y + yy * step;
        float geom = sv.geometry_weight(a, qx, qy, (float)step);
        if (geom <= 0.f) return;
        float4 smp = R::load(input, sv.idx(qx, qy));
        float w = wavelet_kernel(xx) * wavelet_kernel(yy) * geom *
                  expf(-fabsf(luminance(V3{smp.x, smp.y, smp.z}) - lc) / phi);
        sum = sum + V3{smp.x, smp.y, smp.z} * w;
        v += smp.w * smp.w * w * w;
        total += w;
    };
    // Taps in row order.  With feature records (three 128-bit loads a tap)
    // a row's five taps are unrolled so their loads issue together (a-trous
    // 1.12 -> 1.03 ms at 1920x1200); on f32 planes (six loads a tap) the
    // unrolled row needs more registers than it saves (1.08 -> 1.23 ms).
    if constexpr (Sv<G>::kFeatures) {
        for (int32_t yy = -2; yy <= 2; yy++)
#pragma unroll
            for (int32_t xx = -2; xx <= 2; xx++) tap(xx, yy);
    } else {
        for (int32_t yy = -2; yy <= 2; yy++)
            for (int32_t xx = -2; xx <= 2; xx++) tap(xx, yy);
    }
    float dn = wmax(total, .00001f);
    float4 o = make_float4(sum.x / dn, sum.y / dn, sum.z / dn, wmin(sqrtf(v) / dn, 65000.f));
    R::store(out, i, o);
    if (out2) R::store(out2, i, o);
}

template <class G, class R>
__global__ void __launch_bounds__(256) svgf_atrous_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                          const typename R::T* input, typename R::T* out,
                                                          typename R::T* out2, int32_t step) {
    atrous_body<G, R>(f, c, input, out, out2, step, blockIdx.x * blockDim.x + threadIdx.x,
                      blockIdx.y * blockDim.y + threadIdx.y);
}

template <class G, class R, class M>
__global__ void __launch_bounds__(256, 5) svgf_variance_batched(const irt_frame* __restrict__ frames,
                                                             const SView<G>* __restrict__ views,
                                                             const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = svgf_find_view(tile_start, n, blockIdx.x);
    __shared__ __align__(16) irt_frame f;
    __shared__ __align__(16) SView<G> w;
    svgf_stage(frames + v, &f);
    svgf_stage(views + v, &w);
    __syncthreads();
    int32_t x, y;
    svgf_tile_xy(f.size[0], blockIdx.x - __ldg(tile_start + v), x, y);
    typedef typename R::T T;
    variance_body<G, R, M>(f, w.c, (const T*)w.in, (const typename M::T*)w.moments_in, (T*)w.out, x, y);
}

template <class G, class R>
__global__ void __launch_bounds__(256, 5) svgf_atrous_batched(const irt_frame* __restrict__ frames,
                                                           const SView<G>* __restrict__ views,
                                                           const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = svgf_find_view(tile_start, n, blockIdx.x);
    __shared__ __align__(16) irt_frame f;
    __shared__ __align__(16) SView<G> w;
    svgf_stage(frames + v, &f);
    svgf_stage(views + v, &w);
    __syncthreads();
    int32_t x, y;
    svgf_tile_xy(f.size[0], blockIdx.x - __ldg(tile_start + v), x, y);
    typedef typename R::T T;
    atrous_body<G, R>(f, w.c, (const T*)w.in, (T*)w.out, (T*)w.out2, w.step, x, y);
}

template <class G, class R, class M>
static cudaError_t spatial_typed(const SvgfLaunch& L, int stage, cudaStream_t st) {
    SvgfCtx<G> c = make_ctx<G>(L);
    const irt_frame& f = *L.frame;
    typedef typename R::T T;
    if (stage == 1) {
        dim3 block(32, 8);
        dim3 grid((f.size[0] + 31) / 32, (f.size[1] + 7) / 8);
        svgf_variance_kernel<G, R, M><<<grid, block, 0, st>>>(f, c, (const T*)L.in,
                                                              (const typename M::T*)L.moments_in, (T*)L.out);
    } else if (stage == 2) {
        // Blocks of 256 pixels of one row: per 1920x1200 frame (4 passes, f32 / mixed storage)
        // 1.077 / 1.021 ms in 32x8 blocks, 1.062 / 1.018 in 128x2, 1.063 / 1.010 in 64x4,
        // 1.025 / 0.985 in 256x1 (the variance pass is fastest in 32x8: 0.061 against 0.068 ms).
        dim3 block(256, 1);
        dim3 grid((f.size[0] + 255) / 256, f.size[1]);
        svgf_atrous_kernel<G, R><<<grid, block, 0, st>>>(f, c, (const T*)L.in, (T*)L.out, (T*)L.out2, L.step);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class G, class R, class M>
static cudaError_t spatial_batched_typed(const BatchLaunch& B, int stage, cudaStream_t st) {
    const SView<G>* views = static_cast<const SView<G>*>(B.table);
    dim3 block(B.bx, B.by);
    if (stage == 1)
        svgf_variance_batched<G, R, M><<<B.tiles, block, 0, st>>>(B.frames, views, B.tile_start, B.n);
    else if (stage == 2)
        svgf_atrous_batched<G, R><<<B.tiles, block, 0, st>>>(B.frames, views, B.tile_start, B.n);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace irtd

cudaError_t irt_launch_svgf_spatial_batched(const BatchLaunch& B, int stage, cudaStream_t st) {
    using namespace irtd;
    SvgfLaunch L{};
    L.gbuffer.format = B.gbuffer_format;
    L.radiance_f16 = B.radiance_f16;
    L.moments_f16 = stage == 2 ? 0 : B.moments_f16;
    return dispatch_svgf(L, [&](auto g, auto r, auto m) {
        return spatial_batched_typed<decltype(g), decltype(r), decltype(m)>(B, stage, st);
    });
}

cudaError_t irt_launch_svgf_spatial(const SvgfLaunch& L, int stage, cudaStream_t st) {
    using namespace irtd;
    if (stage == 2) {  // a-trous reads no moments
        SvgfLaunch A = L;
        A.moments_f16 = 0;
        return dispatch_svgf(A, [&](auto g, auto r, auto) {
            return spatial_typed<decltype(g), decltype(r), MomF32>(A, stage, st);
        });
    }
    return dispatch_svgf(L, [&](auto g, auto r, auto m) {
        return spatial_typed<decltype(g), decltype(r), decltype(m)>(L, stage, st);
    });
}
