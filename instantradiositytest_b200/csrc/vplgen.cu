// vplgen.cu — CUDA VPL generator (vpl.wgsl:1-47): one thread per VPL path.
// A path starts at a light chosen uniformly (seed salt 7), leaves it along a
// uniform direction of the light's cone (spot) or sphere (point), and at
// each of up to `bounces` surface hits stores the VPL (position, normal,
// flux = source flux x path throughput x BSDF weight / path count), then
// continues with a sampled BSDF direction and Russian roulette between
// rr.x and rr.y.  The reference traces with a hardware ray query against
// the scene's acceleration structure (no face culling); here the ray cast
// runs against the workload's primitive table (dev_prims.cuh).
#include <cuda_runtime.h>

#include "dev_common.cuh"
#include "dev_prims.cuh"
#include "kernels.h"

namespace irtd {

// basis() of common.wgsl:84: columns t, cross(n, t), n.
__device__ __forceinline__ V3 cross3(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ V3 apply_basis(V3 n, V3 v) {
    V3 axis = fabsf(n.z) > .9f ? V3{1.f, 0.f, 0.f} : V3{0.f, 0.f, 1.f};
    V3 t = normalize(cross3(axis, n));
    V3 b = cross3(n, t);
    return t * v.x + b * v.y + n * v.z;
}

// sample_bsdf (common.wgsl:87-97): GGX half-vector lobe with probability
// .25 (dielectric) to .9 (metal), cosine lobe otherwise; weight =
// brdf * cos / mixture pdf.
__device__ __forceinline__ void sample_bsdf(const Surface& s, uint32_t& rng, V3& wi, V3& weight) {
    const V3 wo = s.wo;
    float spec_probability = .25f * (1.f - s.metal) + .9f * s.metal;
    float r2 = s.rough * s.rough;
    float a2 = r2 * r2;
    if (rnd(rng) < spec_probability) {
        float u = rnd(rng);
        float cos_theta = sqrtf((1.f - u) / (1.f + (a2 - 1.f) * u));
        float phi = 2.f * kPI * rnd(rng);
        float st = sqrtf(1.f - cos_theta * cos_theta);
        V3 h = apply_basis(s.n, V3{st * cosf(phi), st * sinf(phi), cos_theta});
        V3 i = -wo;
        wi = i - h * (2.f * dot(h, i));
    } else {
        float u = rnd(rng);
        float phi = 2.f * kPI * rnd(rng);
        wi = apply_basis(s.n, V3{sqrtf(u) * cosf(phi), sqrtf(u) * sinf(phi), sqrtf(1.f - u)});
    }
    float nl = wmax(dot(s.n, wi), 0.f);
    if (nl <= 0.f) {
        weight = V3{0.f, 0.f, 0.f};
        return;
    }
    V3 h = normalize(wo + wi);
    float nh = wmax(dot(s.n, h), 0.f);
    float q = nh * nh * (a2 - 1.f) + 1.f;
    float pdf_d = nl / kPI;
    float pdf_s = a2 * nh / (kPI * q * q * wmax(4.f * fabsf(dot(wo, h)), .00001f));
    float pdf = pdf_d * (1.f - spec_probability) + pdf_s * spec_probability;
    weight = brdf(s, wi) * (nl / wmax(pdf, .00001f));
}

__global__ void __launch_bounds__(128) vpl_kernel(const __grid_constant__ irt_frame f, const irt::PrimTable T,
                                                  const irt_light* lights, irt_vpl* out) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = f.counts[1];
    if (id >= n) return;
    irt_vpl v{};
    const uint32_t n_lights = f.counts[0];
    if (n_lights == 0u) {
        out[id] = v;
        return;
    }
    uint32_t rng = seed(id, 7u, f.size[2]);
    uint32_t light_id = min(to_u32(rnd(rng) * (float)n_lights), n_lights - 1u);
    const irt_light& l = lights[light_id];
    V3 origin = V3{l.position_strength[0], l.position_strength[1], l.position_strength[2]};
    V3 direction;
    float omega = 4.f * kPI;
    if (l.color_type[3] > .5f) {
        float ca = cosf(l.direction_angle[3] * .5f);
        omega = 2.f * kPI * (1.f - ca);
        float u = rnd(rng);
        float z = ca * (1.f - u) + 1.f * u;
        float phi = 2.f * kPI * rnd(rng);
        V3 axis = normalize(V3{l.direction_angle[0], l.direction_angle[1], l.direction_angle[2]});
        float s = sqrtf(1.f - z * z);
        direction = apply_basis(axis, V3{s * cosf(phi), s * sinf(phi), z});
    } else {
        float z = 2.f * rnd(rng) - 1.f;
        float phi = 2.f * kPI * rnd(rng);
        float s = sqrtf(1.f - z * z);
        direction = V3{s * cosf(phi), s * sinf(phi), z};
    }
    V3 color = V3{l.color_type[0], l.color_type[1], l.color_type[2]};
    V3 source_flux = color * (l.position_strength[3] * omega * (float)n_lights);
    V3 throughput = V3{1.f, 1.f, 1.f};
    for (uint32_t bounce = 0; bounce < f.counts[2]; bounce++) {
        float o[3] = {origin.x, origin.y, origin.z}, d[3] = {direction.x, direction.y, direction.z};
        float t, nl[3];
        int k = cast_prims(T, o, d, .0005f, 10000.f, false, t, nl);
        if (k < 0) {
            v.flux[0] = v.flux[1] = v.flux[2] = v.flux[3] = 0.f;
            break;
        }
        const irt::GPrim& p = T.prims[k];
        float w4[4];
        xf4(p.model, nl[0], nl[1], nl[2], 0.f, w4);
        Surface s;
        s.n = normalize(V3{w4[0], w4[1], w4[2]});
        s.p = origin + direction * t;
        s.color = V3{p.color[0], p.color[1], p.color[2]};
        s.rough = p.params[0];
        s.metal = p.params[1];
        V3 wo = -direction;
        if (dot(s.n, wo) <= 0.f) {
            v.flux[0] = v.flux[1] = v.flux[2] = v.flux[3] = 0.f;
            break;
        }
        surface_terms_wo(s, wo);
        v.position[0] = s.p.x;
        v.position[1] = s.p.y;
        v.position[2] = s.p.z;
        v.position[3] = 1.f;
        v.normal[0] = s.n.x;
        v.normal[1] = s.n.y;
        v.normal[2] = s.n.z;
        v.normal[3] = 0.f;
        V3 wi, weight;
        sample_bsdf(s, rng, wi, weight);
        V3 reflected = throughput * weight;
        V3 flux = source_flux * reflected / (float)n;
        v.flux[0] = flux.x;
        v.flux[1] = flux.y;
        v.flux[2] = flux.z;
        v.flux[3] = 0.f;
        if (bounce + 1u >= f.counts[2]) break;
        float survive = wmin(wmax(wmax(reflected.x, wmax(reflected.y, reflected.z)), f.rr[0]), f.rr[1]);
        if (rnd(rng) > survive) break;
        if (luminance(weight) <= 0.f) break;
        throughput = reflected / survive;
        origin = s.p + s.n * .001f;
        direction = wi;
    }
    out[id] = v;
}

}  // namespace irtd

cudaError_t irt_launch_vpls(const VplLaunch& L, cudaStream_t st) {
    const uint32_t n = L.frame->counts[1];
    if (n == 0) return cudaSuccess;
    irtd::vpl_kernel<<<(n + 127) / 128, 128, 0, st>>>(*L.frame, L.prims, L.lights, L.out);
    return cudaGetLastError();
}
