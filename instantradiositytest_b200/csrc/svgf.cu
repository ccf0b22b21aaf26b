// svgf.cu — svgf_temporal (svgf.wgsl:45-76) and the per-pixel position guides
// as sm_100a CUDA.  Built with every f32 operation rounded on its own
// (-fmad=false): the history length `age` is a bilinear average of integers
// that svgf_variance compares with 4, and the positions feed every
// neighbour test, so both follow the reference's arithmetic exactly.
// One thread per pixel in 32x8 blocks.
#include <cuda_runtime.h>

#include "dev_svgf.cuh"
#include "kernels.h"

namespace irtd {

// svgf.wgsl:45-76
// With MomF16 the moment history is (mean, deviation) and the blend of
// history and the current sample is done on central moments (the pooled
// variance of the bilinear taps about their mean, then
// (1-b)*var_h + b*(1-b)*(l - mean_h)^2), which equals the reference's
// E[l^2] - E[l]^2 without its cancellation.
template <class G, class R, class M>
__device__ __forceinline__ void temporal_body(const irt_frame& f, const SvgfCtx<G>& c, const typename R::T* noisy,
                                              const typename R::T* old_radiance, const typename M::T* old_moments,
                                              typename R::T* radiance_out, typename M::T* moments_out, int32_t x,
                                              int32_t y) {
    Sv<G> sv(f, c);
    if (x >= sv.W || y >= sv.H) return;
    size_t i = sv.idx(x, y);
    float4 c4 = R::load(noisy, i);
    V3 cc = V3{c4.x, c4.y, c4.z};
    float l = luminance(cc);
    V3 history = V3{0.f, 0.f, 0.f};
    float hm0 = 0.f, hm1 = 0.f, length_history = 0.f, total = 0.f;
    float tap_w[4] = {0.f, 0.f, 0.f, 0.f}, tap_mean[4], tap_dev[4];  // MomF16 only
    if (c.g.d(i) < 1.f) {
        float2 mv = c.g.mv(i);
        float px = (sv.uvx(x) - mv.x) * (float)sv.W - .5f;
        float py = (sv.uvy(y) - mv.y) * (float)sv.H - .5f;
        float flx = floorf(px), fly = floorf(py);
        int32_t bx = to_i32(flx), by = to_i32(fly);
        float fx = px - flx, fy = py - fly;
        // The pixel's own terms of the 4 history tests, computed once.
        const V3 pa = sv.position(x, y), pn = c.g.n(i);
        const float reach = sv.history_reach(pa);
#pragma unroll
        for (int32_t yy = 0; yy < 2; yy++)
#pragma unroll
            for (int32_t xx = 0; xx < 2; xx++) {
                int32_t qx = bx + xx, qy = by + yy;
                if (!sv.history_ok(pa, pn, reach, qx, qy)) continue;
                size_t q = sv.idx(qx, qy);
                Moments m = M::load(old_moments, q);
                if (m.age <= 0.f) continue;
                float wx = xx == 1 ? fx : 1.f - fx;
                float wy = yy == 1 ? fy : 1.f - fy;
                float w = wx * wy;
                float4 h = R::load(old_radiance, q);
                history = history + V3{h.x, h.y, h.z} * w;
                hm0 += m.mean * w;
                if constexpr (M::central) {
                    tap_w[yy * 2 + xx] = w;
                    tap_mean[yy * 2 + xx] = m.mean;
                    tap_dev[yy * 2 + xx] = m.second;
                } else {
                    hm1 += m.second * w;
                }
                length_history += m.age * w;
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
        if constexpr (M::central) {
            float var_h = 0.f;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (tap_w[k] == 0.f) continue;
                float d = tap_mean[k] - hm0;
                var_h += (tap_dev[k] * tap_dev[k] + d * d) * tap_w[k];
            }
            var_h /= total;
            float d = l - hm0;
            m0 = hm0 * (1.f - beta) + l * beta;
            m1 = var_h * (1.f - beta) + d * d * (beta * (1.f - beta));  // central: the variance
        } else {
            float n0 = hm0 * (1.f - beta) + m0 * beta;
            float n1 = hm1 * (1.f - beta) + m1 * beta;
            m0 = n0;
            m1 = n1;
        }
    } else if constexpr (M::central) {
        m1 = 0.f;
    }
    float variance = M::central ? m1 : wmax(m1 - m0 * m0, 0.f);
    R::store(radiance_out, i, make_float4(result.x, result.y, result.z, wmin(sqrtf(variance), 65000.f)));
    M::store(moments_out, i, Moments{m0, M::central ? sqrtf(variance) : m1, age});
}

// Held to 32 registers (8 blocks of 256, every warp slot of the SM): the pass
// waits on its history and neighbour gathers, and more resident warps hide
// more of that than the spills cost.  Per 1920x1200 frame, f32 / mixed
// storage: 3 blocks by registers (the f16-moments forms take 80) 0.302 /
// 0.394 ms, 4 blocks 0.299 / 0.334, 5 blocks 0.266 / 0.308, 6 blocks 0.266 /
// 0.290, 8 blocks 0.254 / 0.296 ms.
template <class G, class R, class M>
__global__ void __launch_bounds__(256, 8) svgf_temporal_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ SvgfCtx<G> c,
                                                            const typename R::T* noisy, const typename R::T* old_radiance,
                                                            const typename M::T* old_moments, typename R::T* radiance_out,
                                                            typename M::T* moments_out) {
    temporal_body<G, R, M>(f, c, noisy, old_radiance, old_moments, radiance_out, moments_out,
                           blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

template <class G, class R, class M>
__global__ void __launch_bounds__(256, 8) svgf_temporal_batched(const irt_frame* __restrict__ frames,
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
    temporal_body<G, R, M>(f, w.c, (const T*)w.in, (const T*)w.aux, (const typename M::T*)w.moments_in, (T*)w.out,
                           (typename M::T*)w.moments_out, x, y);
}

// World position of every pixel, world(pixel_uv, depth, inv_vp)
// (common.wgsl:46-47) with its f32 operations rounded one by one, and in w
// the SVGF pixel scale distance(position, camera) / height (svgf.wgsl:30), or
// -1 where depth >= 1.  The lighting and SVGF kernels read positions from
// here instead of recomputing them per neighbour tap.
// With `previous` set, the same for the previous frame's depth and
// previous_inv_vp (the positions history_valid / history_ok compare with).
__device__ __forceinline__ void guide_body(const irt_frame& f, const float* depth, int previous, float4* out, size_t i) {
    const uint32_t W = f.size[0];
    if (i >= (size_t)W * f.size[1]) return;
    uint32_t x = (uint32_t)(i % W), y = (uint32_t)(i / W);
    float d = __ldg(depth + i);
    V3 p = world(((float)x + .5f) / (float)W, ((float)y + .5f) / (float)f.size[1], d,
                 previous ? f.previous_inv_vp : f.inv_vp);
    float s = d < 1.f ? distance(p, V3{f.camera[0], f.camera[1], f.camera[2]}) / (float)f.size[1] : -1.f;
    out[i] = make_float4(p.x, p.y, p.z, s);
}

__global__ void __launch_bounds__(256) guide_kernel(const __grid_constant__ irt_frame f, const float* depth,
                                                    int previous, float4* out) {
    guide_body(f, depth, previous, out, (size_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// Guide of this frame and the decoded edge-stopping features of every pixel:
// feat[2i] = (normal, roughness), feat[2i+1] = (colour, metal).
template <class G>
__device__ __forceinline__ void feature_body(const irt_frame& f, const G& g, float4* guide, float4* feat, size_t i) {
    guide_body(f, g.depth, 0, guide, i);
    if (i >= (size_t)f.size[0] * f.size[1]) return;
    V3 n = g.n(i), c = g.c(i);
    float2 pm = g.pm(i);
    feat[2 * i] = make_float4(n.x, n.y, n.z, pm.x);
    feat[2 * i + 1] = make_float4(c.x, c.y, c.z, pm.y);
}

template <class G>
__global__ void __launch_bounds__(256) feature_kernel(const __grid_constant__ irt_frame f, const __grid_constant__ G g,
                                                      float4* guide, float4* feat) {
    feature_body<G>(f, g, guide, feat, (size_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// Batched guides (in = depth, out = guide) and depth/normal history copy
// (in = depth, aux = normal, out = previous depth, out2 = previous normal);
// 1-D tiles of 256 pixels.
template <class G>
__global__ void __launch_bounds__(256) guide_batched(const irt_frame* __restrict__ frames, const SView<G>* __restrict__ views,
                                                     const uint32_t* __restrict__ tile_start, uint32_t n, int previous) {
    const uint32_t v = svgf_find_view(tile_start, n, blockIdx.x);
    const SView<G>& w = views[v];
    guide_body(frames[v], (const float*)w.in, previous, (float4*)w.out,
               (size_t)(blockIdx.x - __ldg(tile_start + v)) * blockDim.x + threadIdx.x);
}

template <class G>
__global__ void __launch_bounds__(256) feature_batched(const irt_frame* __restrict__ frames,
                                                       const SView<G>* __restrict__ views,
                                                       const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = svgf_find_view(tile_start, n, blockIdx.x);
    const SView<G>& w = views[v];
    feature_body<G>(frames[v], w.c.g, (float4*)w.out, (float4*)w.out2,
                    (size_t)(blockIdx.x - __ldg(tile_start + v)) * blockDim.x + threadIdx.x);
}

template <class G>
__global__ void __launch_bounds__(256) history_batched(const irt_frame* __restrict__ frames, const SView<G>* __restrict__ views,
                                                       const uint32_t* __restrict__ tile_start, uint32_t n) {
    const uint32_t v = svgf_find_view(tile_start, n, blockIdx.x);
    const SView<G>& w = views[v];
    const irt_frame& f = frames[v];
    const size_t i = (size_t)(blockIdx.x - __ldg(tile_start + v)) * blockDim.x + threadIdx.x;
    if (i >= (size_t)f.size[0] * f.size[1]) return;
    ((float*)w.out)[i] = ((const float*)w.in)[i];
    typedef typename G::NormalT N;
    ((N*)w.out2)[i] = ((const N*)w.aux)[i];
}

template <class G, class R, class M>
static cudaError_t svgf_typed(const SvgfLaunch& L, int stage, cudaStream_t st) {
    SvgfCtx<G> c = make_ctx<G>(L);
    const irt_frame& f = *L.frame;
    typedef typename R::T T;
    dim3 block(32, 8);
    dim3 grid((f.size[0] + 31) / 32, (f.size[1] + 7) / 8);
    switch (stage) {
    case 0:
        svgf_temporal_kernel<G, R, M><<<grid, block, 0, st>>>(f, c, (const T*)L.in, (const T*)L.aux,
                                                              (const typename M::T*)L.moments_in, (T*)L.out,
                                                              (typename M::T*)L.moments_out);
        break;
    case 3:
    case 4: {
        size_t P = (size_t)f.size[0] * f.size[1];
        guide_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(f, stage == 3 ? L.gbuffer.depth : L.old_depth,
                                                                   stage == 4, (float4*)L.out);
    } break;
    case 6: {
        size_t P = (size_t)f.size[0] * f.size[1];
        feature_kernel<G><<<(unsigned)((P + 255) / 256), 256, 0, st>>>(f, c.g, (float4*)L.out, (float4*)L.out2);
    } break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class G, class R, class M>
static cudaError_t svgf_batched_typed(const BatchLaunch& B, int stage, cudaStream_t st) {
    const SView<G>* views = static_cast<const SView<G>*>(B.table);
    switch (stage) {
    case 0: svgf_temporal_batched<G, R, M><<<B.tiles, dim3(B.bx, B.by), 0, st>>>(B.frames, views, B.tile_start, B.n); break;
    case 3:
    case 4: guide_batched<G><<<B.tiles, 256, 0, st>>>(B.frames, views, B.tile_start, B.n, stage == 4); break;
    case 5: history_batched<G><<<B.tiles, 256, 0, st>>>(B.frames, views, B.tile_start, B.n); break;
    case 6: feature_batched<G><<<B.tiles, 256, 0, st>>>(B.frames, views, B.tile_start, B.n); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace irtd

size_t irt_svgf_view_size(int gbuffer_format) {
    using namespace irtd;
    switch (gbuffer_format) {
    case IRT_GBUFFER_F32: return sizeof(SView<GbF32>);
    case IRT_GBUFFER_F16: return sizeof(SView<GbF16>);
    default: return sizeof(SView<GbPacked>);
    }
}

template <class G>
static void fill_view(const SvgfLaunch& L, void* out) {
    using namespace irtd;
    SView<G> w;
    w.c = make_ctx<G>(L);
    w.in = L.in;
    w.aux = L.aux;
    w.moments_in = L.moments_in;
    w.out = L.out;
    w.out2 = L.out2;
    w.moments_out = L.moments_out;
    w.step = L.step;
    *static_cast<SView<G>*>(out) = w;
}

void irt_svgf_view_fill(const SvgfLaunch& L, void* out) {
    using namespace irtd;
    switch (L.gbuffer.format) {
    case IRT_GBUFFER_F32: fill_view<GbF32>(L, out); break;
    case IRT_GBUFFER_F16: fill_view<GbF16>(L, out); break;
    default: fill_view<GbPacked>(L, out); break;
    }
}

cudaError_t irt_launch_svgf_batched(const BatchLaunch& B, int stage, cudaStream_t st) {
    using namespace irtd;
    if (B.n == 0) return cudaSuccess;
    if (stage == 1 || stage == 2) return irt_launch_svgf_spatial_batched(B, stage, st);
    SvgfLaunch L{};
    L.gbuffer.format = B.gbuffer_format;
    L.radiance_f16 = B.radiance_f16;
    L.moments_f16 = B.moments_f16;
    return dispatch_svgf(L, [&](auto g, auto r, auto m) {
        return svgf_batched_typed<decltype(g), decltype(r), decltype(m)>(B, stage, st);
    });
}

cudaError_t irt_launch_svgf(const SvgfLaunch& L, int stage, cudaStream_t st) {
    using namespace irtd;
    if (stage == 1 || stage == 2) return irt_launch_svgf_spatial(L, stage, st);
    if (stage == 3 || stage == 4)  // guides read neither radiance nor moments
        return svgf_typed<GbF32, RadF32, MomF32>(L, stage, st);
    if (stage == 6) {  // features read the G-buffer format only
        SvgfLaunch F = L;
        F.radiance_f16 = 0;
        F.moments_f16 = 0;
        return dispatch_svgf(F, [&](auto g, auto, auto) {
            return svgf_typed<decltype(g), RadF32, MomF32>(F, stage, st);
        });
    }
    return dispatch_svgf(L, [&](auto g, auto r, auto m) {
        return svgf_typed<decltype(g), decltype(r), decltype(m)>(L, stage, st);
    });
}
