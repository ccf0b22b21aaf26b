// dev_common.cuh — device restatement of the per-pixel math of common.wgsl and
// lighting.wgsl (helpers, BRDF, light/VPL evaluation, reservoir algebra) and
// the G-buffer / radiance storage formats.
//
// Precision: IEEE f32 with correctly rounded division and square root;
// transcendental functions are CUDA's accurate versions (cosf, sinf, powf,
// expf).  inverseSqrt(x) is evaluated as 1/sqrt(x).  The integer RNG is
// bit-exact with common.wgsl:39-44.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/irt.h"

namespace irtd {

// The ray queue of the march holds 2*W*H records: one class of shadow rays
// fills it from the front (counter [0]), the other from the back (counter
// [2]); the march takes the [0] + [2] rays in queue order, queue position i
// being record slot ray_slot(i).
__device__ __forceinline__ uint32_t ray_slot(uint32_t i, uint32_t front, uint32_t cap) {
    return i < front ? i : cap - 1u - (i - front);
}

// ------------------------------------------------------------------ float3
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float distance(V3 a, V3 b) { return length(a - b); }
__device__ __forceinline__ V3 normalize(V3 a) { return a / sqrtf(dot(a, a)); }
// WGSL max/min on ordinary (non-NaN) values.
__device__ __forceinline__ float wmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float wmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ V3 vmax(V3 a, V3 b) { return {wmax(a.x, b.x), wmax(a.y, b.y), wmax(a.z, b.z)}; }
__device__ __forceinline__ V3 vmin(V3 a, V3 b) { return {wmin(a.x, b.x), wmin(a.y, b.y), wmin(a.z, b.z)}; }
__device__ __forceinline__ float wclamp(float e, float lo, float hi) { return wmin(wmax(e, lo), hi); }
__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ V3 xyz(float4 v) { return V3{v.x, v.y, v.z}; }

constexpr float kPI = 3.14159265359f;

// WGSL f32 -> i32 / u32 conversions saturate (NaN -> 0).
__device__ __forceinline__ int32_t to_i32(float v) { return __float2int_rz(v); }
__device__ __forceinline__ uint32_t to_u32(float v) { return __float2uint_rz(v); }

// Column-major mat4 (WGSL mat4x4 / glam::Mat4) times (x, y, z, w).
__device__ __forceinline__ void mat_vec(const irt_mat4& m, float x, float y, float z, float w, float out[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) out[r] = m.m[0 * 4 + r] * x + m.m[1 * 4 + r] * y + m.m[2 * 4 + r] * z + m.m[3 * 4 + r] * w;
}

// ------------------------------------------------------------------ RNG
// common.wgsl:39-43 (PCG-RXS-M-XS output of an LCG state).
__device__ __forceinline__ float rnd(uint32_t& state) {
    state = state * 747796405u + 2891336453u;
    uint32_t w = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return __uint2float_rn((w >> 22u) ^ w) * (1.0f / 4294967296.0f);
}
// common.wgsl:44
__device__ __forceinline__ uint32_t seed(uint32_t i, uint32_t salt, uint32_t frame_index) {
    return i * 1973u + frame_index * 9277u + salt * 26699u + 89173u;
}
__device__ __forceinline__ float luminance(V3 c) { return c.x * .2126f + c.y * .7152f + c.z * .0722f; }
// common.wgsl:46
__device__ __forceinline__ V3 world(float u, float v, float depth, const irt_mat4& m) {
    float h[4];
    mat_vec(m, u * 2.f - 1.f, 1.f - v * 2.f, depth, 1.f, h);
    return V3{h[0] / h[3], h[1] / h[3], h[2] / h[3]};
}

// A shading point and the BRDF terms that depend only on it and the camera
// (computed once per pixel, the same values brdf() would compute per call).
struct Surface {
    V3 p, n, color;
    float rough, metal;
    V3 wo;            // normalize(camera - p)
    float nv, a2, g1v, km;
    V3 f0;            // mix(vec3(.04), color, metal)
};
// The same for an explicit outgoing direction (a VPL path vertex: -ray).
__device__ __forceinline__ void surface_terms_wo(Surface& s, V3 wo) {
    s.wo = wo;
    s.nv = wmax(dot(s.n, s.wo), .00001f);
    float a = s.rough * s.rough;
    s.a2 = a * a;
    s.g1v = 2.f * s.nv / (s.nv + sqrtf(s.a2 + (1.f - s.a2) * s.nv * s.nv));
    s.km = 1.f - s.metal;
    s.f0 = V3{.04f * s.km + s.color.x * s.metal, .04f * s.km + s.color.y * s.metal, .04f * s.km + s.color.z * s.metal};
}
__device__ __forceinline__ void surface_terms(Surface& s, V3 camera) {
    s.wo = normalize(camera - s.p);
    s.nv = wmax(dot(s.n, s.wo), .00001f);
    float a = s.rough * s.rough;
    s.a2 = a * a;
    s.g1v = 2.f * s.nv / (s.nv + sqrtf(s.a2 + (1.f - s.a2) * s.nv * s.nv));
    s.km = 1.f - s.metal;
    s.f0 = V3{.04f * s.km + s.color.x * s.metal, .04f * s.km + s.color.y * s.metal, .04f * s.km + s.color.z * s.metal};
}

// Divisions of the shading functions below (brdf, direct, indirect): the
// approximate divide (reciprocal and multiply, within 2 ulp; WGSL's own f32
// division is specified to 2.5 ulp) instead of the IEEE sequence; every
// denominator here is bounded below and far from the reciprocal's range
// limit.  The visibility march keeps its own build's division.
__device__ __forceinline__ float sdiv(float a, float b) { return __fdividef(a, b); }

// common.wgsl:67-74 (GGX with Smith G1 terms plus Lambert, F0 = mix(.04, c, metal))
// toward wi for the surface's view direction; (1 - vh)^5 by multiplication.
__device__ __forceinline__ V3 brdf(const Surface& s, V3 wi) {
    const V3 wo = s.wo;
    const float nv = s.nv;
    float nl = wmax(dot(s.n, wi), 0.f);
    if (nl <= 0.f) return V3{0.f, 0.f, 0.f};
    V3 h = normalize(wo + wi);
    float nh = wmax(dot(s.n, h), 0.f);
    float vh = wmax(dot(wo, h), 0.f);
    const float a2 = s.a2;
    float q = nh * nh * (a2 - 1.f) + 1.f;
    float d = sdiv(a2, kPI * q * q);
    float g1l = sdiv(2.f * nl, nl + sqrtf(a2 + (1.f - a2) * nl * nl));
    const float km = s.km;
    const V3 f0 = s.f0;
    float x = 1.f - vh;
    float x2 = x * x;
    float p5 = x2 * x2 * x;
    V3 fr = V3{f0.x + (1.f - f0.x) * p5, f0.y + (1.f - f0.y) * p5, f0.z + (1.f - f0.z) * p5};
    float den = wmax(4.f * nv * nl, .00001f);
    float spec = sdiv(d * s.g1v * g1l, den);
    V3 out;
    out.x = sdiv((1.f - fr.x) * km * s.color.x, kPI) + fr.x * spec;
    out.y = sdiv((1.f - fr.y) * km * s.color.y, kPI) + fr.y * spec;
    out.z = sdiv((1.f - fr.z) * km * s.color.z, kPI) + fr.z * spec;
    return out;
}

// Light and VPL records as three 16-byte vectors (read-only cache loads).
// Lights are read from the per-frame prepared copy (prepare_lights_kernel):
// da holds the normalised spot direction and cos(angle / 2) instead of the
// raw direction and angle — the two values direct() derives per call.
struct DLight {
    float4 ps, da, ct;  // position_strength, (normalised direction, cos half angle), color_type
};
struct DVpl {
    float4 pos, nrm, flux;
};
__device__ __forceinline__ DLight load_light(const irt_light* base, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(base + i);
    return DLight{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}
__device__ __forceinline__ DVpl load_vpl(const irt_vpl* base, size_t i) {
    const float4* p = reinterpret_cast<const float4*>(base + i);
    return DVpl{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// Prepared light: the spot direction normalised and cos(angle / 2).
__device__ __forceinline__ DLight prepare_light(const irt_light& l) {
    V3 d = normalize(V3{l.direction_angle[0], l.direction_angle[1], l.direction_angle[2]});
    DLight o;
    o.ps = make_float4(l.position_strength[0], l.position_strength[1], l.position_strength[2], l.position_strength[3]);
    o.da = make_float4(d.x, d.y, d.z, cosf(l.direction_angle[3] * .5f));
    o.ct = make_float4(l.color_type[0], l.color_type[1], l.color_type[2], l.color_type[3]);
    return o;
}

// common.wgsl:75-79
__device__ __forceinline__ V3 direct(const Surface& s, const DLight& l) {
    V3 delta = xyz(l.ps) - s.p;
    float r2 = wmax(dot(delta, delta), .0001f);
    V3 wi = delta * sdiv(1.f, sqrtf(r2));
    if (l.ct.w > 0.5f && dot(-wi, xyz(l.da)) < l.da.w) return V3{0.f, 0.f, 0.f};
    V3 b = brdf(s, wi);
    float nl = wmax(dot(s.n, wi), 0.f);
    float st = l.ps.w;
    return V3{sdiv(b.x * nl * l.ct.x * st, r2), sdiv(b.y * nl * l.ct.y * st, r2), sdiv(b.z * nl * l.ct.z * st, r2)};
}

// common.wgsl:80-83
__device__ __forceinline__ V3 indirect(const Surface& s, const DVpl& v) {
    V3 delta = xyz(v.pos) - s.p;
    float r2 = wmax(dot(delta, delta), .0025f);
    V3 wi = delta * sdiv(1.f, sqrtf(r2));
    V3 b = brdf(s, wi);
    float nl = wmax(dot(s.n, wi), 0.f);
    float ne = wmax(dot(xyz(v.nrm), -wi), 0.f);
    float den = 4.f * kPI * r2;
    return V3{sdiv(b.x * nl * ne * v.flux.x, den), sdiv(b.y * nl * ne * v.flux.y, den),
              sdiv(b.z * nl * ne * v.flux.z, den)};
}

// ------------------------------------------------------------------ reservoirs
struct Res {
    uint32_t id, source, count, age;
    float sum, target, pdf;
    uint32_t generation;
};
__device__ __forceinline__ Res res_load(const irt_reservoir* base, size_t i) {
    const uint4* p = reinterpret_cast<const uint4*>(base + i);
    uint4 a = __ldg(p), b = __ldg(p + 1);
    return Res{a.x, a.y, a.z, a.w, __uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z), b.w};
}
// A reservoir is one 32-byte sector, moved as two 128-bit accesses.
__device__ __forceinline__ void res_store(irt_reservoir* base, size_t i, const Res& r) {
    uint4* p = reinterpret_cast<uint4*>(base + i);
    p[0] = make_uint4(r.id, r.source, r.count, r.age);
    p[1] = make_uint4(__float_as_uint(r.sum), __float_as_uint(r.target), __float_as_uint(r.pdf), r.generation);
}
// common.wgsl:98
__device__ __forceinline__ Res res_empty(const irt_frame& f) {
    return Res{0u, f.size[2], 0u, 0u, 0.f, 0.f, 0.f, f.size[3]};
}
// common.wgsl:99
__device__ __forceinline__ float normalization(const Res& r) {
    if (r.count == 0u || r.target <= 0.f) return 0.f;
    return r.sum / ((float)r.count * r.target);
}
// common.wgsl:100-106 — the random draw happens only for an accepted weight.
__device__ __forceinline__ void res_add(Res& r, uint32_t id, uint32_t source, float target, float pdf, float weight,
                                        uint32_t count, uint32_t age, uint32_t& rng) {
    r.count += count;
    if (weight <= 0.f || weight > 1e30f) return;
    r.sum += weight;
    if (rnd(rng) * r.sum < weight) {
        r.id = id;
        r.source = source;
        r.target = target;
        r.pdf = pdf;
        r.age = age;
    }
}
// lighting.wgsl:51
__device__ __forceinline__ Res cap(Res a, uint32_t limit) {
    if (a.count > limit) {
        a.sum *= (float)limit / (float)a.count;
        a.count = limit;
    }
    return a;
}

// ------------------------------------------------------------------ G-buffer formats
// F32: float4 normal/colour, float2 params/motion.
struct GbF32 {
    const float* depth;
    const float4* normal;
    const float4* color;
    const float2* params;
    const float2* motion;
    typedef float4 NormalT;
    __device__ __forceinline__ float d(size_t i) const { return __ldg(depth + i); }
    __device__ __forceinline__ V3 n(size_t i) const { return xyz(__ldg(normal + i)); }
    __device__ __forceinline__ V3 c(size_t i) const { return xyz(__ldg(color + i)); }
    __device__ __forceinline__ float2 pm(size_t i) const { return __ldg(params + i); }
    __device__ __forceinline__ float2 mv(size_t i) const { return __ldg(motion + i); }
    __device__ __forceinline__ static V3 decode_normal(NormalT v) { return xyz(v); }
};

__device__ __forceinline__ V3 half4_xyz(uint2 v) {
    __half2 a = *reinterpret_cast<__half2*>(&v.x);
    __half2 b = *reinterpret_cast<__half2*>(&v.y);
    return V3{__low2float(a), __high2float(a), __low2float(b)};
}
__device__ __forceinline__ float2 half2_f2(uint32_t v) {
    __half2 a = *reinterpret_cast<__half2*>(&v);
    return make_float2(__low2float(a), __high2float(a));
}

// F16: the reference's Rgba16Float / Rg16Float targets.
struct GbF16 {
    const float* depth;
    const uint2* normal;
    const uint2* color;
    const uint32_t* params;
    const uint32_t* motion;
    typedef uint2 NormalT;
    __device__ __forceinline__ float d(size_t i) const { return __ldg(depth + i); }
    __device__ __forceinline__ V3 n(size_t i) const { return half4_xyz(__ldg(normal + i)); }
    __device__ __forceinline__ V3 c(size_t i) const { return half4_xyz(__ldg(color + i)); }
    __device__ __forceinline__ float2 pm(size_t i) const { return half2_f2(__ldg(params + i)); }
    __device__ __forceinline__ float2 mv(size_t i) const { return half2_f2(__ldg(motion + i)); }
    __device__ __forceinline__ static V3 decode_normal(NormalT v) { return half4_xyz(v); }
};

// PACKED: octahedral snorm16x2 normal, rgba8 colour, f16 params/motion.
__device__ __forceinline__ V3 oct_decode(uint32_t v) {
    float x = fmaxf((float)(int16_t)(v & 0xffffu) / 32767.f, -1.f);
    float y = fmaxf((float)(int16_t)(v >> 16) / 32767.f, -1.f);
    float z = 1.f - fabsf(x) - fabsf(y);
    float t = fmaxf(-z, 0.f);
    x += x >= 0.f ? -t : t;
    y += y >= 0.f ? -t : t;
    float inv = 1.f / sqrtf(x * x + y * y + z * z);
    return V3{x * inv, y * inv, z * inv};
}
struct GbPacked {
    const float* depth;
    const uint32_t* normal;
    const uint32_t* color;
    const uint32_t* params;
    const uint32_t* motion;
    typedef uint32_t NormalT;
    __device__ __forceinline__ float d(size_t i) const { return __ldg(depth + i); }
    __device__ __forceinline__ V3 n(size_t i) const { return oct_decode(__ldg(normal + i)); }
    __device__ __forceinline__ V3 c(size_t i) const {
        uint32_t v = __ldg(color + i);
        return V3{(float)(v & 255u) / 255.f, (float)((v >> 8) & 255u) / 255.f, (float)((v >> 16) & 255u) / 255.f};
    }
    __device__ __forceinline__ float2 pm(size_t i) const { return half2_f2(__ldg(params + i)); }
    __device__ __forceinline__ float2 mv(size_t i) const { return half2_f2(__ldg(motion + i)); }
    __device__ __forceinline__ static V3 decode_normal(NormalT v) { return oct_decode(v); }
};

// ------------------------------------------------------------------ radiance formats
struct RadF32 {
    typedef float4 T;
    __device__ __forceinline__ static float4 load(const T* p, size_t i) { return p[i]; }
    __device__ __forceinline__ static void store(T* p, size_t i, float4 v) { p[i] = v; }
    __device__ __forceinline__ static float quant(float v) { return v; }
};
struct RadF16 {
    typedef uint2 T;
    __device__ __forceinline__ static float4 load(const T* p, size_t i) {
        uint2 v = p[i];
        __half2 a = *reinterpret_cast<__half2*>(&v.x);
        __half2 b = *reinterpret_cast<__half2*>(&v.y);
        return make_float4(__low2float(a), __high2float(a), __low2float(b), __high2float(b));
    }
    __device__ __forceinline__ static void store(T* p, size_t i, float4 v) {
        __half2 a = __floats2half2_rn(v.x, v.y);
        __half2 b = __floats2half2_rn(v.z, v.w);
        uint2 o;
        o.x = *reinterpret_cast<uint32_t*>(&a);
        o.y = *reinterpret_cast<uint32_t*>(&b);
        p[i] = o;
    }
    __device__ __forceinline__ static float quant(float v) { return __half2float(__float2half_rn(v)); }
};

// ------------------------------------------------------------------ device error word
#define IRT_DEVERR_BVH_ESCAPE 1u  // an escape link did not advance the cursor
#define IRT_DEVERR_BVH_BUDGET 2u  // node visits exceeded 2N-1 per query
__device__ __forceinline__ void raise_error(uint32_t* err, uint32_t code) {
    if (err) atomicOr(err, code);
}

// The checked build (IRT_CHECKED=1, libirt_checked.so): every index a kernel
// takes from data rather than from its thread position — reservoir ids into
// the light table, gathers at reprojected or neighbouring pixels, ray-queue
// slots and the output slots in the ray records, leaf-cache object ids — is
// tested against its table before the access.  An index out of range sets
// IRT_DEVERR_INDEX in the session's error word and the access is skipped, so
// a bad index is reported instead of faulting (the role compute-sanitizer
// would play).  In the default build the test compiles away: these indices
// are in range by construction.
#ifndef IRT_CHECKED
#define IRT_CHECKED 0
#endif
#define IRT_DEVERR_INDEX 4u  // checked build: an index outside its table
__device__ __forceinline__ bool index_ok(uint32_t* err, uint64_t i, uint64_t n) {
#if IRT_CHECKED
    if (i >= n) {
        raise_error(err, IRT_DEVERR_INDEX);
        return false;
    }
#else
    (void)err;
    (void)i;
    (void)n;
#endif
    return true;
}

}  // namespace irtd
