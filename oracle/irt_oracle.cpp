// irt_oracle.cpp — CPU restatement of the reference's lighting hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py (its
// cpu_baseline leg and its `--impl reference` arm) load it, and only as the
// checker or the CPU reference arm; the product path (libirt.so) never links
// or calls it.
//
// It restates, function by function, the WGSL of the reference:
//   common.wgsl:31-47, :67-83, :98-106   (sample_field, random, seed,
//                                         luminance, world, pixel_uv, brdf,
//                                         direct, indirect, reservoir ops)
//   lighting.wgsl:22-134                 (the 8 lighting entry points)
//   sdf.wgsl:1-81                        (distance bounds, BVH walk, march)
//   svgf.wgsl:18-110                     (SVGF temporal, variance, a-trous)
// and the host pass schedule of src/renderer.rs:1873-1960 and
// src/svgf.rs:140-261.
//
// Precision modes: T = float evaluates every f32 operation of the WGSL in
// IEEE binary32 with no contraction (built with -ffp-contract=off); T = double
// evaluates the same operations in binary64 ("FP64 transcription") while the
// integer RNG stays u32.  Storage rounding to binary16 happens exactly where
// the session stores Rgba16Float (radiance format F16), with
// round-to-nearest-even like the `half` crate 2.7.1 the reference uses.
// Parity pin: the reference has no runnable golden outputs here (Rust and
// Vulkan are absent); the oracle is pinned by the reference's CPU known-answer
// tests (src/math.rs, src/renderer.rs, src/settings.rs), restated in tests/.

#include "../include/irt.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------- binary16
uint16_t f32_to_f16_rne(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xffu;
    uint32_t man = x & 0x7fffffu;
    if (exp == 0xffu) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u : 0u));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t mid = 1u << (shift - 1u);
        if (rem > mid || (rem == mid && (half & 1u))) half++;
        return (uint16_t)(sign | half);
    }
    uint32_t half = sign | ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) half++;
    return (uint16_t)half;
}

float f16_to_f32(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) {
            x = sign;
        } else {
            int e = -1;
            do {
                e++;
                man <<= 1;
            } while (!(man & 0x400u));
            x = sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3ffu) << 13);
        }
    } else if (exp == 31) {
        x = sign | 0x7f800000u | (man << 13);
    } else {
        x = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

float round_f16(float v) { return f16_to_f32(f32_to_f16_rne(v)); }

// ---------------------------------------------------------------- vectors
template <class T>
struct V3 {
    T x, y, z;
};
template <class T> V3<T> v3(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> T distance(V3<T> a, V3<T> b) { return length(a - b); }
template <class T> V3<T> normalize(V3<T> a) { return a / std::sqrt(dot(a, a)); }
template <class T> T fmax_(T a, T b) { return a > b ? a : b; }  // WGSL max on non-NaN
template <class T> T fmin_(T a, T b) { return a < b ? a : b; }
template <class T> V3<T> vmax(V3<T> a, V3<T> b) { return {fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)}; }
template <class T> V3<T> vmin(V3<T> a, V3<T> b) { return {fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)}; }
template <class T> T clampv(T e, T lo, T hi) { return fmin_(fmax_(e, lo), hi); }
template <class T> V3<T> ld3(const float* p) { return {(T)p[0], (T)p[1], (T)p[2]}; }

// Column-major mat4 times (x, y, z, w), WGSL `m * vec4`.
template <class T>
void mat_vec(const irt_mat4& m, T x, T y, T z, T w, T out[4]) {
    for (int r = 0; r < 4; r++)
        out[r] = (T)m.m[0 * 4 + r] * x + (T)m.m[1 * 4 + r] * y + (T)m.m[2 * 4 + r] * z +
                 (T)m.m[3 * 4 + r] * w;
}

// WGSL f32 -> i32 conversion saturates.
template <class T> int32_t to_i32(T v) {
    if (!(v == v)) return 0;
    if (v >= (T)2147483647.0) return 2147483647;
    if (v <= (T)-2147483648.0) return (int32_t)0x80000000u;
    return (int32_t)v;
}
template <class T> uint32_t to_u32(T v) {
    if (!(v > (T)0)) return 0u;
    if (v >= (T)4294967295.0) return 0xffffffffu;
    return (uint32_t)v;
}

template <class T> T PI_() { return (T)3.14159265359; }

// ---------------------------------------------------------------- inputs
struct Scene {
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    const irt_light* lights;
    const float* atlas;  // dequantised texels, x fastest
    uint32_t dims[3];
    int field_linear = 0;  // 1: the reference's hardware-filtered sample_field (weights rounded to the
                           // nearest 1/256), 2: the same with weights truncated to 1/256
};

struct GBuffer {  // F32 layout
    const float* depth;
    const float* normal;  // 4 per texel
    const float* color;   // 4
    const float* params;  // 2
    const float* motion;  // 2
};

struct Counters {
    uint64_t march_steps = 0, nodes = 0, box_queries = 0, field_queries = 0, rays = 0, evals = 0;
};

// ---------------------------------------------------------------- the path
template <class T>
struct Path {
    const irt_frame& f;
    const Scene& sc;
    const GBuffer& g;
    const irt_vpl* current_vpls;
    const irt_vpl* previous_vpls;
    const irt_vpl* archived_vpls;
    Counters* ctr;
    uint32_t W, H;

    Path(const irt_frame& frame, const Scene& scene, const GBuffer& gb, const irt_vpl* cur,
         const irt_vpl* prev, const irt_vpl* arch, Counters* c)
        : f(frame), sc(scene), g(gb), current_vpls(cur), previous_vpls(prev), archived_vpls(arch),
          ctr(c), W(frame.size[0]), H(frame.size[1]) {}

    // common.wgsl:39-43
    static T random(uint32_t& state) {
        state = state * 747796405u + 2891336453u;
        uint32_t w = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
        return (T)(float_from_u32((w >> 22u) ^ w)) * ((T)1.0 / (T)4294967296.0);
    }
    // u32 -> f32 conversion (round to nearest) in FP32; exact in FP64.
    static T float_from_u32(uint32_t v) { return (T)v; }
    // common.wgsl:44
    uint32_t seed(uint32_t i, uint32_t salt) const {
        return i * 1973u + f.size[2] * 9277u + salt * 26699u + 89173u;
    }
    static T luminance(V3<T> c) { return c.x * (T).2126 + c.y * (T).7152 + c.z * (T).0722; }
    // common.wgsl:46
    V3<T> world(T u, T v, T depth, const irt_mat4& m) const {
        T h[4];
        mat_vec<T>(m, u * (T)2 - (T)1, (T)1 - v * (T)2, depth, (T)1, h);
        return v3(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
    }
    // common.wgsl:47
    void pixel_uv(uint32_t x, uint32_t y, T& u, T& v) const {
        u = ((T)x + (T).5) / (T)W;
        v = ((T)y + (T).5) / (T)H;
    }
    V3<T> camera() const { return v3((T)f.camera[0], (T)f.camera[1], (T)f.camera[2]); }

    struct Surface {
        V3<T> p, n, color;
        T rough, metal;
    };

    // common.wgsl:67-74
    V3<T> brdf(const Surface& s, V3<T> wo, V3<T> wi) const {
        T nv = fmax_(dot(s.n, wo), (T).00001);
        T nl = fmax_(dot(s.n, wi), (T)0);
        if (nl <= (T)0) return v3<T>(0, 0, 0);
        V3<T> h = normalize(wo + wi);
        T nh = fmax_(dot(s.n, h), (T)0);
        T vh = fmax_(dot(wo, h), (T)0);
        T a = s.rough * s.rough;
        T a2 = a * a;
        T q = nh * nh * (a2 - (T)1) + (T)1;
        T d = a2 / (PI_<T>() * q * q);
        T g1v = (T)2 * nv / (nv + std::sqrt(a2 + ((T)1 - a2) * nv * nv));
        T g1l = (T)2 * nl / (nl + std::sqrt(a2 + ((T)1 - a2) * nl * nl));
        // mix(vec3(.04), color, metal) = .04*(1-metal) + color*metal
        V3<T> f0 = v3((T).04 * ((T)1 - s.metal) + s.color.x * s.metal,
                      (T).04 * ((T)1 - s.metal) + s.color.y * s.metal,
                      (T).04 * ((T)1 - s.metal) + s.color.z * s.metal);
        T p5 = std::pow((T)1 - vh, (T)5);
        V3<T> fr = v3(f0.x + ((T)1 - f0.x) * p5, f0.y + ((T)1 - f0.y) * p5, f0.z + ((T)1 - f0.z) * p5);
        T spec_den = fmax_((T)4 * nv * nl, (T).00001);
        T diff_k = (T)1 - s.metal;
        V3<T> out;
        out.x = ((T)1 - fr.x) * diff_k * s.color.x / PI_<T>() + fr.x * d * g1v * g1l / spec_den;
        out.y = ((T)1 - fr.y) * diff_k * s.color.y / PI_<T>() + fr.y * d * g1v * g1l / spec_den;
        out.z = ((T)1 - fr.z) * diff_k * s.color.z / PI_<T>() + fr.z * d * g1v * g1l / spec_den;
        return out;
    }
    // common.wgsl:75-79
    V3<T> direct(const Surface& s, uint32_t id) const {
        if (ctr) ctr->evals++;
        const irt_light& l = sc.lights[id];
        V3<T> delta = ld3<T>(l.position_strength) - s.p;
        T r2 = fmax_(dot(delta, delta), (T).0001);
        V3<T> wi = delta * ((T)1 / std::sqrt(r2));
        if ((T)l.color_type[3] > (T)0.5 &&
            dot(-wi, normalize(ld3<T>(l.direction_angle))) < std::cos((T)l.direction_angle[3] * (T).5))
            return v3<T>(0, 0, 0);
        V3<T> b = brdf(s, normalize(camera() - s.p), wi);
        T nl = fmax_(dot(s.n, wi), (T)0);
        V3<T> c = ld3<T>(l.color_type);
        T strength = (T)l.position_strength[3];
        return v3(b.x * nl * c.x * strength / r2, b.y * nl * c.y * strength / r2,
                  b.z * nl * c.z * strength / r2);
    }
    // common.wgsl:80-83
    V3<T> indirect(const Surface& s, const irt_vpl& v) const {
        if (ctr) ctr->evals++;
        V3<T> delta = ld3<T>(v.position) - s.p;
        T r2 = fmax_(dot(delta, delta), (T).0025);
        V3<T> wi = delta * ((T)1 / std::sqrt(r2));
        V3<T> b = brdf(s, normalize(camera() - s.p), wi);
        T nl = fmax_(dot(s.n, wi), (T)0);
        T ne = fmax_(dot(ld3<T>(v.normal), -wi), (T)0);
        V3<T> fl = ld3<T>(v.flux);
        T den = (T)4 * PI_<T>() * r2;
        return v3(b.x * nl * ne * fl.x / den, b.y * nl * ne * fl.y / den, b.z * nl * ne * fl.z / den);
    }

    // Reservoir in T precision (stored back as f32).
    struct Res {
        uint32_t id, source, count, age;
        T sum, target, pdf;
        uint32_t generation;
    };
    static Res load(const irt_reservoir& r) {
        return Res{r.id, r.source, r.count, r.age, (T)r.sum, (T)r.selected_target, (T)r.pdf, r.generation};
    }
    static irt_reservoir store(const Res& r) {
        irt_reservoir o;
        o.id = r.id;
        o.source = r.source;
        o.count = r.count;
        o.age = r.age;
        o.sum = (float)r.sum;
        o.selected_target = (float)r.target;
        o.pdf = (float)r.pdf;
        o.generation = r.generation;
        return o;
    }
    // common.wgsl:98
    Res empty() const { return Res{0u, f.size[2], 0u, 0u, (T)0, (T)0, (T)0, f.size[3]}; }
    // common.wgsl:99
    static T normalization(const Res& r) {
        if (r.count == 0u || r.target <= (T)0) return (T)0;
        return r.sum / ((T)r.count * r.target);
    }
    // common.wgsl:100-106
    static bool add(Res& r, uint32_t id, uint32_t source, T target, T pdf, T weight, uint32_t count,
                    uint32_t age, uint32_t& rng) {
        r.count += count;
        if (weight <= (T)0 || weight > (T)1e30) return false;
        r.sum += weight;
        if (random(rng) * r.sum < weight) {
            r.id = id;
            r.source = source;
            r.target = target;
            r.pdf = pdf;
            r.age = age;
            return true;
        }
        return false;
    }
    // lighting.wgsl:51
    static Res cap(Res a, uint32_t limit) {
        if (a.count > limit) {
            a.sum *= (T)limit / (T)a.count;
            a.count = limit;
        }
        return a;
    }

    // ---------------------------------------------------- G-buffer access
    T depth_at(uint32_t x, uint32_t y) const { return (T)g.depth[(size_t)y * W + x]; }
    V3<T> normal_at(uint32_t x, uint32_t y) const { return ld3<T>(g.normal + ((size_t)y * W + x) * 4); }
    V3<T> color_at(uint32_t x, uint32_t y) const { return ld3<T>(g.color + ((size_t)y * W + x) * 4); }
    T param_at(uint32_t x, uint32_t y, int c) const { return (T)g.params[((size_t)y * W + x) * 2 + c]; }
    T motion_at(uint32_t x, uint32_t y, int c) const { return (T)g.motion[((size_t)y * W + x) * 2 + c]; }

    // lighting.wgsl:30-34
    Surface surface(uint32_t x, uint32_t y) const {
        Surface s;
        T u, v;
        pixel_uv(x, y, u, v);
        s.p = world(u, v, depth_at(x, y), f.inv_vp);
        s.n = normalize(normal_at(x, y));
        s.color = color_at(x, y);
        s.rough = param_at(x, y, 0);
        s.metal = param_at(x, y, 1);
        return s;
    }
    bool valid(uint32_t x, uint32_t y) const { return depth_at(x, y) < (T)1; }
    // lighting.wgsl:36-40
    bool compatible(const Surface& a, uint32_t qx, uint32_t qy) const {
        T d = depth_at(qx, qy);
        if (d >= (T)1) return false;
        T u, v;
        pixel_uv(qx, qy, u, v);
        V3<T> p = world(u, v, d, f.inv_vp);
        V3<T> n = normalize(normal_at(qx, qy));
        return dot(a.n, n) > (T)f.temporal[2] &&
               distance(a.p, p) < (T)f.temporal[1] * fmax_(distance(a.p, camera()), (T)1);
    }
    // lighting.wgsl:41-44
    void reproject(uint32_t x, uint32_t y, int32_t& qx, int32_t& qy) const {
        T u, v;
        pixel_uv(x, y, u, v);
        u = u - motion_at(x, y, 0);
        v = v - motion_at(x, y, 1);
        qx = to_i32(std::floor(u * (T)W));
        qy = to_i32(std::floor(v * (T)H));
    }
    // lighting.wgsl:45-50
    bool history_valid(const Surface& a, int32_t qx, int32_t qy, const float* prev_depth,
                       const float* prev_normal) const {
        if (f.flags[0] == 0u || f.flags[1] != f.size[3] || qx < 0 || qy < 0 || qx >= (int32_t)W ||
            qy >= (int32_t)H)
            return false;
        size_t qi = (size_t)qy * W + (size_t)qx;
        T d = (T)prev_depth[qi];
        if (d >= (T)1) return false;
        V3<T> oldp = world(((T)qx + (T).5) / (T)W, ((T)qy + (T).5) / (T)H, d, f.previous_inv_vp);
        V3<T> pn = ld3<T>(prev_normal + qi * 4);
        return dot(a.n, pn) > (T)f.temporal[2] &&
               distance(a.p, oldp) < (T)f.temporal[1] * fmax_(distance(a.p, camera()), (T)1);
    }
    // lighting.wgsl:22-24
    bool vpl_sample_valid(const Res& r) const {
        return r.generation == f.size[3] && r.target > (T)0 && r.id < f.counts[1] &&
               f.size[2] - r.source <= to_u32((T)f.rr[2]);
    }
    // lighting.wgsl:25-29
    const irt_vpl& selected_vpl(const Res& r) const {
        if (r.source == f.size[2]) return current_vpls[r.id];
        if (r.source + 1u == f.size[2]) return previous_vpls[r.id];
        uint32_t slots = to_u32((T)f.rr[2]) + 1u;
        return archived_vpls[(size_t)(r.source % slots) * f.counts[1] + r.id];
    }
    // lighting.wgsl:86-89
    void neighbor(uint32_t x, uint32_t y, uint32_t& rng, int32_t& qx, int32_t& qy) const {
        T angle = (T)2 * PI_<T>() * random(rng);
        T radius = std::sqrt(random(rng)) * (T)f.restir[3];
        qx = (int32_t)x + to_i32(std::nearbyint(std::cos(angle) * radius));
        qy = (int32_t)y + to_i32(std::nearbyint(std::sin(angle) * radius));
    }

    // ---------------------------------------------------- sdf.wgsl
    static T signed_box_distance(V3<T> p, V3<T> lo, V3<T> hi) {
        V3<T> delta = vmax(lo - p, p - hi);
        return length(vmax(delta, v3<T>(0, 0, 0))) + fmin_(fmax_(delta.x, fmax_(delta.y, delta.z)), (T)0);
    }
    T texel(uint32_t x, uint32_t y, uint32_t z) const {
        return (T)sc.atlas[((size_t)z * sc.dims[1] + y) * sc.dims[0] + x];
    }
    // The reference's filtered variant of sample_field (src/renderer.rs:
    // 277-286): textureSampleLevel(fields, field_sampler,
    // (vec3(origin) + q + .5) / vec3(dims), 0.) through a clamp-to-edge
    // linear sampler, i.e. at texel coordinate x = origin + q + .5.  The
    // filter is restated from the linear-filtering formula of the CUDA C++
    // Programming Guide ("Texture Fetching" appendix), which the device
    // sampler implements: x_B = x - 0.5, i = floor(x_B) and alpha = frac(x_B)
    // held in 9-bit fixed point with 8 fractional bits, and the value is the
    // sum over the 8 texels of (1 - alpha or alpha) products per axis,
    // clamped to the atlas edge.  Weighted in the same z, y, x order as
    // sample_field.  The guide leaves the rounding of alpha and the
    // arithmetic precision of the filter open: mode 1 rounds alpha to the
    // nearest 1/256, mode 2 truncates it — two readings of the same
    // documented filter, whose distance bounds what the documentation pins.
    T linear_field(const uint32_t origin[3], V3<T> q) const {
        const T qa[3] = {q.x, q.y, q.z};
        int64_t i0[3];
        T alpha[3];
        for (int a = 0; a < 3; a++) {
            const T x = ((T)origin[a] + qa[a]) + (T).5;
            const double xb = (double)x - 0.5;
            const double fl = std::floor(xb);
            i0[a] = (int64_t)fl;
            const double f256 = (xb - fl) * 256.0;
            alpha[a] = (T)((sc.field_linear == 2 ? std::floor(f256) : std::floor(f256 + 0.5)) / 256.0);
        }
        auto at = [&](int a, int64_t i) {
            return (uint32_t)std::min<int64_t>(std::max<int64_t>(i, 0), (int64_t)sc.dims[a] - 1);
        };
        T value = 0;
        for (uint32_t z = 0; z < 2; z++)
            for (uint32_t y = 0; y < 2; y++)
                for (uint32_t x = 0; x < 2; x++) {
                    T wx = x == 1 ? alpha[0] : (T)1 - alpha[0];
                    T wy = y == 1 ? alpha[1] : (T)1 - alpha[1];
                    T wz = z == 1 ? alpha[2] : (T)1 - alpha[2];
                    value += texel(at(0, i0[0] + x), at(1, i0[1] + y), at(2, i0[2] + z)) * wx * wy * wz;
                }
        return value;
    }
    // common.wgsl:31-38
    T sample_field(const uint32_t origin[3], V3<T> q, uint32_t res) const {
        if (sc.field_linear) return linear_field(origin, q);
        uint32_t cx = std::min(to_u32(std::floor(q.x)), res - 2u);
        uint32_t cy = std::min(to_u32(std::floor(q.y)), res - 2u);
        uint32_t cz = std::min(to_u32(std::floor(q.z)), res - 2u);
        V3<T> fr = v3(q.x - (T)cx, q.y - (T)cy, q.z - (T)cz);
        T value = 0;
        for (uint32_t z = 0; z < 2; z++)
            for (uint32_t y = 0; y < 2; y++)
                for (uint32_t x = 0; x < 2; x++) {
                    T wx = x == 1 ? fr.x : (T)1 - fr.x;
                    T wy = y == 1 ? fr.y : (T)1 - fr.y;
                    T wz = z == 1 ? fr.z : (T)1 - fr.z;
                    value += texel(origin[0] + cx + x, origin[1] + cy + y, origin[2] + cz + z) * wx * wy * wz;
                }
        return value;
    }
    // sdf.wgsl:5-33
    T mesh_distance(V3<T> p, const irt_mesh& m) const {
        T geometry_bound = signed_box_distance(p, ld3<T>(m.geometry_lo), ld3<T>(m.geometry_hi));
        if ((T)m.geometry_lo[3] > (T).5) {
            if (ctr) ctr->box_queries++;
            return geometry_bound;
        }
        if (ctr) ctr->field_queries++;
        uint32_t res = m.field[3];
        V3<T> lo = ld3<T>(m.lo), hi = ld3<T>(m.hi);
        V3<T> clamped = vmin(vmax(p, lo), hi);
        V3<T> q = (clamped - lo) * ld3<T>(m.grid);
        T value = sample_field(m.field, q, res);
        T bound = value - (T)m.grid[3] * ((T).5 + (T)1 / (T)128);
        V3<T> outside = vmax(vmax(lo - p, p - hi), v3<T>(0, 0, 0));
        T os = dot(outside, outside);
        if (os > (T)0) {
            T positive = fmax_(bound, (T)0);
            bound = std::sqrt(positive * positive + os);
        }
        if (bound > (T)0) bound *= (T)m.geometry_hi[3];
        T sphere_bound = length(p - ld3<T>(m.enclosing_sphere)) - (T)m.enclosing_sphere[3];
        return fmax_(bound, fmax_(geometry_bound, sphere_bound));
    }
    // sdf.wgsl:35-41
    void object_distance(V3<T> p, uint32_t id, bool need_spacing, T& d, T& voxel) const {
        const irt_object& obj = sc.objects[id];
        const irt_mesh& mesh = sc.meshes[obj.info[0]];
        T h[4];
        mat_vec<T>(obj.inverse, p.x, p.y, p.z, (T)1, h);
        V3<T> local = v3(h[0], h[1], h[2]);
        float scale, spacing;
        std::memcpy(&scale, &obj.info[2], 4);
        std::memcpy(&spacing, &obj.info[3], 4);
        d = mesh_distance(local, mesh) * (T)scale;
        if (d > (T)0) d *= (T).9999;
        voxel = need_spacing ? (T)spacing : (T)f.sdf[1];
    }
    // sdf.wgsl:42-60
    void scene_distance(V3<T> p, bool need_spacing, uint32_t hint, T& best, T& voxel,
                        uint32_t& closest) const {
        best = (T)1e20;
        voxel = (T)f.sdf[1];
        closest = hint;
        uint32_t cursor = 0;
        uint32_t n = f.counts[3];
        if (hint < n) object_distance(p, hint, need_spacing, best, voxel);
        uint32_t end = n * 2u - 1u;
        while (cursor < end) {
            if (ctr) ctr->nodes++;
            const irt_node& node = sc.nodes[cursor];
            V3<T> delta = vmax(vmax(ld3<T>(node.lo) - p, p - ld3<T>(node.hi)), v3<T>(0, 0, 0));
            V3<T> lb = delta * (T).9998;
            T b = fmax_(best, (T)0);
            if (dot(lb, lb) > b * b) {
                cursor = node.info[3];
                continue;
            }
            if (node.info[2] == 1u) {
                if (node.info[0] != hint) {
                    T d, vx;
                    object_distance(p, node.info[0], need_spacing, d, vx);
                    if (d < best) {
                        best = d;
                        voxel = vx;
                        closest = node.info[0];
                    }
                }
            }
            cursor++;
        }
    }
    // sdf.wgsl:61-81
    T visibility(V3<T> p, V3<T> n, V3<T> target, V3<T> end_normal) const {
        if (ctr) ctr->rays++;
        T eps = (T)f.sdf[1];
        T best, voxel;
        uint32_t closest;
        scene_distance(p, true, 0xffffffffu, best, voxel, closest);
        T epsilon = fmax_(eps, voxel * (T).65);
        V3<T> origin = p + n * epsilon;
        V3<T> endpoint = target;
        if (dot(end_normal, end_normal) > (T).5) {
            T b2, v2;
            uint32_t c2;
            scene_distance(target, true, 0xffffffffu, b2, v2, c2);
            endpoint = endpoint + end_normal * fmax_(eps, v2 * (T).65);
        }
        V3<T> delta = endpoint - origin;
        T limit = length(delta) - eps;
        if (limit <= (T)0) return (T)1;
        V3<T> direction = normalize(delta);
        T t = eps;
        T result = 1;
        T previous = (T)1e20;
        uint32_t steps = to_u32((T)f.sdf[0]);
        for (uint32_t i = 0; i < steps; i++) {
            if (t >= limit) return clampv(result, (T)0, (T)1);
            if (ctr) ctr->march_steps++;
            T h, vx;
            scene_distance(origin + direction * t, false, closest, h, vx, closest);
            if (h < eps) return (T)0;
            T y = h * h / ((T)2 * previous);
            T d = std::sqrt(fmax_(h * h - y * y, (T)0));
            if (t > y) result = fmin_(result, (T)f.sdf[2] * d / (t - y));
            if (result < (T).001) return (T)0;
            previous = h;
            t += h;
        }
        return (T)0;
    }
};

// ---------------------------------------------------------------- state
struct State {
    uint32_t W = 0, H = 0, vpl_count = 0, max_history = 0;
    int precision = 0;      // 0 = FP32, 1 = FP64
    int radiance_f16 = 0;   // Rgba16Float storage points
    int field_filter = 0;   // 1: hardware-filtered sample_field (src/renderer.rs:277-286)
    int threads = 0;
    // Rows [row0, row1) that the passes evaluate (the whole image unless a
    // timing sample restricts it to a band).
    uint32_t row0 = 0, row1 = 0xffffffffu;
    std::vector<irt_reservoir> res[2][3];  // [direct/indirect][0..2]
    std::vector<irt_vpl> archive;
    std::vector<float> prev_depth, prev_normal;
    std::vector<float> direct_lighting, lighting;
    std::vector<float> moments[2], feedback[2], temporal, scratch[2], histories[2];
    Counters last;
};

inline float store_rad(const State& st, float v) { return st.radiance_f16 ? round_f16(v) : v; }

template <class T>
void lighting_passes(State& st, const irt_frame& f, const Scene& sc, const GBuffer& g,
                     const irt_vpl* cur, const irt_vpl* prev, int first_pass, int last_pass) {
    const uint32_t W = st.W, H = st.H;
    const size_t P = (size_t)W * H;
    typedef typename Path<T>::Res Res;
    typedef typename Path<T>::Surface Surface;
    Counters total;
    // Archive ring (src/renderer.rs:1873-1884).
    if (first_pass <= 0 && last_pass >= 0) {
        uint32_t slot = f.size[2] % (st.max_history + 1u);
        std::copy(cur, cur + st.vpl_count, st.archive.begin() + (size_t)slot * st.vpl_count);
    }
    // Pass schedule of src/renderer.rs:1889-1928: candidates -> [0],
    // temporal [0]+history[2] -> [1], spatial [1] -> [2], resolve reads [2].
    for (int pass = 0; pass < 8; pass++) {
        if (pass < first_pass || pass > last_pass) continue;
        uint64_t steps = 0, nodes = 0, boxq = 0, fieldq = 0, rays = 0, evals = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(st.threads) \
    reduction(+ : steps, nodes, boxq, fieldq, rays, evals)
        for (int64_t yy = (int64_t)st.row0; yy < (int64_t)std::min(H, st.row1); yy++) {
            Counters c;
            Path<T> path(f, sc, g, cur, prev, st.archive.data(), &c);
            uint32_t y = (uint32_t)yy;
            for (uint32_t x = 0; x < W; x++) {
                uint32_t id = y * W + x;
                switch (pass) {
                case 0: {  // candidates_direct, lighting.wgsl:52-58
                    Res r = path.empty();
                    uint32_t rng = path.seed(id, 11u);
                    if (path.valid(x, y) && f.counts[0] > 0u) {
                        Surface s = path.surface(x, y);
                        T pdf = (T)1 / (T)f.counts[0];
                        for (uint32_t i = 0; i < f.restir[0]; i++) {
                            uint32_t lid = std::min(to_u32(Path<T>::random(rng) * (T)f.counts[0]), f.counts[0] - 1u);
                            T target = Path<T>::luminance(path.direct(s, lid));
                            Path<T>::add(r, lid, f.size[2], target, pdf, target / pdf, 1u, 0u, rng);
                        }
                    }
                    st.res[0][0][id] = Path<T>::store(r);
                } break;
                case 1: {  // candidates_indirect, lighting.wgsl:59-65
                    Res r = path.empty();
                    uint32_t rng = path.seed(id, 13u);
                    if (path.valid(x, y)) {
                        Surface s = path.surface(x, y);
                        T pdf = (T)1 / (T)f.counts[1];
                        for (uint32_t i = 0; i < f.restir[1]; i++) {
                            uint32_t vid = std::min(to_u32(Path<T>::random(rng) * (T)f.counts[1]), f.counts[1] - 1u);
                            const irt_vpl& v = cur[vid];
                            T target = Path<T>::luminance(path.indirect(s, v));
                            Path<T>::add(r, vid, f.size[2], target, pdf, target / pdf, 1u, 0u, rng);
                        }
                    }
                    st.res[1][0][id] = Path<T>::store(r);
                } break;
                case 2:
                case 3: {  // temporal_direct / temporal_indirect, lighting.wgsl:66-85
                    int dom = pass - 2;
                    Res r = Path<T>::load(st.res[dom][0][id]);
                    int32_t qx, qy;
                    path.reproject(x, y, qx, qy);
                    uint32_t rng = path.seed(id, dom == 0 ? 17u : 19u);
                    if (path.valid(x, y)) {
                        Surface s = path.surface(x, y);
                        if (path.history_valid(s, qx, qy, st.prev_depth.data(), st.prev_normal.data())) {
                            uint32_t limit = to_u32((T)f.rr[2]) * f.restir[dom];
                            Res previous = Path<T>::cap(
                                Path<T>::load(st.res[dom][2][(size_t)qy * W + (size_t)qx]), limit);
                            if (dom == 0) {
                                if (previous.generation == f.size[3] && previous.target > (T)0 &&
                                    previous.id < f.counts[0] && previous.age < to_u32((T)f.rr[2])) {
                                    T target = Path<T>::luminance(path.direct(s, previous.id));
                                    Path<T>::add(r, previous.id, previous.source, target, previous.pdf,
                                                 target * Path<T>::normalization(previous) * (T)previous.count,
                                                 previous.count, previous.age + 1u, rng);
                                }
                            } else if (path.vpl_sample_valid(previous)) {
                                const irt_vpl& v = path.selected_vpl(previous);
                                T target = Path<T>::luminance(path.indirect(s, v));
                                Path<T>::add(r, previous.id, previous.source, target, previous.pdf,
                                             target * Path<T>::normalization(previous) * (T)previous.count,
                                             previous.count, previous.age + 1u, rng);
                            }
                        }
                    }
                    st.res[dom][1][id] = Path<T>::store(r);
                } break;
                case 4:
                case 5: {  // spatial_direct / spatial_indirect, lighting.wgsl:90-105
                    int dom = pass - 4;
                    Res r = Path<T>::load(st.res[dom][1][id]);
                    uint32_t rng = path.seed(id, dom == 0 ? 23u : 29u);
                    if (path.valid(x, y)) {
                        Surface s = path.surface(x, y);
                        for (uint32_t i = 0; i < f.restir[2]; i++) {
                            int32_t qx, qy;
                            path.neighbor(x, y, rng, qx, qy);
                            if (qx < 0 || qy < 0 || qx >= (int32_t)W || qy >= (int32_t)H) continue;
                            if (!path.compatible(s, (uint32_t)qx, (uint32_t)qy)) continue;
                            Res previous = Path<T>::load(st.res[dom][1][(size_t)qy * W + (size_t)qx]);
                            if (dom == 0) {
                                if (previous.target > (T)0) {
                                    T target = Path<T>::luminance(path.direct(s, previous.id));
                                    Path<T>::add(r, previous.id, previous.source, target, previous.pdf,
                                                 target * Path<T>::normalization(previous) * (T)previous.count,
                                                 previous.count, previous.age, rng);
                                }
                            } else if (path.vpl_sample_valid(previous)) {
                                T target = Path<T>::luminance(path.indirect(s, path.selected_vpl(previous)));
                                Path<T>::add(r, previous.id, previous.source, target, previous.pdf,
                                             target * Path<T>::normalization(previous) * (T)previous.count,
                                             previous.count, previous.age, rng);
                            }
                        }
                    }
                    uint32_t limit = to_u32((T)f.rr[2]) * f.restir[dom] * 8u;
                    st.res[dom][2][id] = Path<T>::store(Path<T>::cap(r, limit));
                } break;
                case 6: {  // resolve_direct, lighting.wgsl:106-122
                    V3<T> result = v3<T>(0, 0, 0);
                    if (path.valid(x, y)) {
                        Surface s = path.surface(x, y);
                        Res d = Path<T>::load(st.res[0][2][id]);
                        uint32_t dbg = f.flags[2];
                        if (d.target > (T)0 && dbg != 2u && dbg < 3u) {
                            V3<T> value = path.direct(s, d.id);
                            if (Path<T>::luminance(value) > (T)0) {
                                T vis = path.visibility(s.p, s.n, ld3<T>(sc.lights[d.id].position_strength),
                                                        v3<T>(0, 0, 0));
                                T k = Path<T>::normalization(d);
                                result = result + v3(value.x * k * vis, value.y * k * vis, value.z * k * vis);
                            }
                        }
                        if (dbg == 3u) result = s.color;
                        if (dbg == 4u) result = v3(s.n.x * (T).5 + (T).5, s.n.y * (T).5 + (T).5, s.n.z * (T).5 + (T).5);
                        if (dbg == 5u) {
                            T mx = path.motion_at(x, y, 0), my = path.motion_at(x, y, 1);
                            result = v3(clampv((T).5 + mx * (T)50, (T)0, (T)1), clampv((T).5 + my * (T)50, (T)0, (T)1), (T).5);
                        }
                    }
                    float* o = &st.direct_lighting[(size_t)id * 4];
                    o[0] = (float)result.x;
                    o[1] = (float)result.y;
                    o[2] = (float)result.z;
                    o[3] = 1.f;
                } break;
                case 7: {  // resolve_indirect, lighting.wgsl:123-134
                    const float* dl = &st.direct_lighting[(size_t)id * 4];
                    V3<T> result = v3((T)dl[0], (T)dl[1], (T)dl[2]);
                    uint32_t dbg = f.flags[2];
                    if (path.valid(x, y) && dbg != 1u && dbg < 3u) {
                        Res v = Path<T>::load(st.res[1][2][id]);
                        if (path.vpl_sample_valid(v)) {
                            Surface s = path.surface(x, y);
                            const irt_vpl& smp = path.selected_vpl(v);
                            V3<T> value = path.indirect(s, smp);
                            if (Path<T>::luminance(value) > (T)0) {
                                T vis = path.visibility(s.p, s.n, ld3<T>(smp.position), ld3<T>(smp.normal));
                                T k = Path<T>::normalization(v);
                                result = result + v3(value.x * k * vis, value.y * k * vis, value.z * k * vis);
                            }
                        }
                    }
                    float* o = &st.lighting[(size_t)id * 4];
                    o[0] = store_rad(st, (float)fmin_(result.x, (T)65000));
                    o[1] = store_rad(st, (float)fmin_(result.y, (T)65000));
                    o[2] = store_rad(st, (float)fmin_(result.z, (T)65000));
                    o[3] = 1.f;
                } break;
                }
            }
            steps += c.march_steps;
            nodes += c.nodes;
            boxq += c.box_queries;
            fieldq += c.field_queries;
            rays += c.rays;
            evals += c.evals;
        }
        total.march_steps += steps;
        total.nodes += nodes;
        total.box_queries += boxq;
        total.field_queries += fieldq;
        total.rays += rays;
        total.evals += evals;
    }
    (void)P;
    st.last = total;
}

// ---------------------------------------------------------------- SVGF
template <class T>
struct Svgf {
    const irt_frame& f;
    const GBuffer& g;
    const float* old_depth;
    const float* old_normal;
    int32_t W, H;
    Svgf(const irt_frame& fr, const GBuffer& gb, const float* od, const float* on)
        : f(fr), g(gb), old_depth(od), old_normal(on), W((int32_t)fr.size[0]), H((int32_t)fr.size[1]) {}

    static T lum(V3<T> c) { return Path<T>::luminance(c); }
    size_t idx(int32_t x, int32_t y) const { return (size_t)y * (size_t)W + (size_t)x; }
    V3<T> camera() const { return v3((T)f.camera[0], (T)f.camera[1], (T)f.camera[2]); }
    bool inside(int32_t x, int32_t y) const { return x >= 0 && y >= 0 && x < W && y < H; }
    V3<T> world(T u, T v, T depth, const irt_mat4& m) const {
        T h[4];
        mat_vec<T>(m, u * (T)2 - (T)1, (T)1 - v * (T)2, depth, (T)1, h);
        return v3(h[0] / h[3], h[1] / h[3], h[2] / h[3]);
    }
    T uvx(int32_t x) const { return ((T)(uint32_t)x + (T).5) / (T)W; }
    T uvy(int32_t y) const { return ((T)(uint32_t)y + (T).5) / (T)H; }
    // svgf.wgsl:19
    V3<T> position(int32_t x, int32_t y) const { return world(uvx(x), uvy(y), (T)g.depth[idx(x, y)], f.inv_vp); }
    V3<T> normal(int32_t x, int32_t y) const { return ld3<T>(g.normal + idx(x, y) * 4); }
    V3<T> color(int32_t x, int32_t y) const { return ld3<T>(g.color + idx(x, y) * 4); }
    // svgf.wgsl:20-26
    bool history_ok(int32_t px, int32_t py, int32_t qx, int32_t qy) const {
        if (f.flags[0] == 0u || f.flags[1] != f.size[3] || !inside(qx, qy)) return false;
        T d = (T)old_depth[idx(qx, qy)];
        if (d >= (T)1) return false;
        V3<T> a = position(px, py);
        V3<T> b = world(uvx(qx), uvy(qy), d, f.previous_inv_vp);
        return distance(a, b) < (T)f.temporal[1] * fmax_(distance(a, camera()), (T)1) &&
               dot(normal(px, py), ld3<T>(old_normal + idx(qx, qy) * 4)) > (T)f.temporal[2];
    }
    struct Guide {
        V3<T> position, normal, color;
        T m0, m1, pixel_scale;
    };
    // svgf.wgsl:28-31
    Guide guide(int32_t x, int32_t y) const {
        Guide a;
        a.position = position(x, y);
        a.normal = normal(x, y);
        a.color = color(x, y);
        a.m0 = (T)g.params[idx(x, y) * 2];
        a.m1 = (T)g.params[idx(x, y) * 2 + 1];
        a.pixel_scale = distance(a.position, camera()) / (T)f.size[1];
        return a;
    }
    // svgf.wgsl:32-44
    T geometry_weight(const Guide& a, int32_t qx, int32_t qy, T stride) const {
        if (!inside(qx, qy) || (T)g.depth[idx(qx, qy)] >= (T)1) return (T)0;
        V3<T> nq = normal(qx, qy);
        T wn = std::pow(fmax_(dot(a.normal, nq), (T)0), (T)64);
        V3<T> wq = position(qx, qy);
        T tolerance = fmax_((T).0001, a.pixel_scale * stride * (T).5);
        T wz = std::exp(-std::fabs(dot(wq - a.position, a.normal)) / tolerance);
        V3<T> dc = a.color - color(qx, qy);
        T dm0 = a.m0 - (T)g.params[idx(qx, qy) * 2];
        T dm1 = a.m1 - (T)g.params[idx(qx, qy) * 2 + 1];
        T wc = std::exp(-length(dc) * (T)8 - std::sqrt(dm0 * dm0 + dm1 * dm1) * (T)8);
        return wn * wz * wc;
    }
};

template <class T>
void svgf_passes(State& st, const irt_frame& f, const GBuffer& g, uint32_t iterations) {
    const int32_t W = (int32_t)st.W, H = (int32_t)st.H;
    const int current = (int)(f.size[2] % 2u), old = 1 - current;
    const size_t P = (size_t)W * (size_t)H;
    if (f.flags[2] >= 3u) {  // src/svgf.rs:154-161
        st.histories[current] = st.lighting;
        return;
    }
    Svgf<T> sv(f, g, st.prev_depth.data(), st.prev_normal.data());
    const float* noisy = st.lighting.data();
    auto rgb = [](const float* img, size_t i) { return v3((T)img[i * 4], (T)img[i * 4 + 1], (T)img[i * 4 + 2]); };
    // svgf_temporal (svgf.wgsl:45-76): noisy + feedback[old] + moments[old].
    {
        const float* old_rad = st.feedback[old].data();
        const float* old_mom = st.moments[old].data();
        float* rad_out = st.temporal.data();
        float* mom_out = st.moments[current].data();
#pragma omp parallel for schedule(dynamic, 4) num_threads(st.threads)
        for (int32_t y = (int32_t)st.row0; y < (int32_t)std::min((uint32_t)H, st.row1); y++)
            for (int32_t x = 0; x < W; x++) {
                size_t i = sv.idx(x, y);
                V3<T> c = rgb(noisy, i);
                T l = Svgf<T>::lum(c);
                V3<T> history = v3<T>(0, 0, 0);
                T hm0 = 0, hm1 = 0, length_history = 0, total = 0;
                if ((T)g.depth[i] < (T)1) {
                    T px = (((T)(uint32_t)x + (T).5) / (T)W - (T)g.motion[i * 2]) * (T)W - (T).5;
                    T py = (((T)(uint32_t)y + (T).5) / (T)H - (T)g.motion[i * 2 + 1]) * (T)H - (T).5;
                    T flx = std::floor(px), fly = std::floor(py);
                    int32_t bx = to_i32(flx), by = to_i32(fly);
                    T fx = px - flx, fy = py - fly;
                    for (int32_t yy = 0; yy < 2; yy++)
                        for (int32_t xx = 0; xx < 2; xx++) {
                            int32_t qx = bx + xx, qy = by + yy;
                            if (!sv.history_ok(x, y, qx, qy)) continue;
                            size_t q = sv.idx(qx, qy);
                            const float* m = old_mom + q * 4;
                            if ((T)m[2] <= (T)0) continue;
                            T wx = xx == 1 ? fx : (T)1 - fx;
                            T wy = yy == 1 ? fy : (T)1 - fy;
                            T w = wx * wy;
                            history = history + rgb(old_rad, q) * w;
                            hm0 += (T)m[0] * w;
                            hm1 += (T)m[1] * w;
                            length_history += (T)m[2] * w;
                            total += w;
                        }
                }
                T age = 1;
                V3<T> result = c;
                T m0 = l, m1 = l * l;
                if (total > (T).001) {
                    history = history / total;
                    hm0 /= total;
                    hm1 /= total;
                    age = fmin_(length_history / total + (T)1, (T)f.temporal[3]);
                    T lo = (T)1e20, hi = 0;
                    typename Svgf<T>::Guide a = sv.guide(x, y);
                    for (int32_t yy = -1; yy <= 1; yy++)
                        for (int32_t xx = -1; xx <= 1; xx++) {
                            int32_t qx = std::min(std::max(x + xx, 0), W - 1);
                            int32_t qy = std::min(std::max(y + yy, 0), H - 1);
                            if (sv.geometry_weight(a, qx, qy, (T)1) > (T).01) {
                                T v = Svgf<T>::lum(rgb(noisy, sv.idx(qx, qy)));
                                lo = fmin_(lo, v);
                                hi = fmax_(hi, v);
                            }
                        }
                    T lh = Svgf<T>::lum(history);
                    T scale = clampv(lh, lo * (T).5, hi * (T)1.5 + (T).001) / fmax_(lh, (T).000001);
                    history = history * scale;
                    T alpha = fmax_((T)1 - (T)f.temporal[0], (T)1 / age);
                    // mix(history, c, alpha) = history*(1-alpha) + c*alpha
                    result = v3(history.x * ((T)1 - alpha) + c.x * alpha, history.y * ((T)1 - alpha) + c.y * alpha,
                                history.z * ((T)1 - alpha) + c.z * alpha);
                    T beta = fmax_((T).2, (T)1 / age);
                    T n0 = hm0 * ((T)1 - beta) + m0 * beta;
                    T n1 = hm1 * ((T)1 - beta) + m1 * beta;
                    m0 = n0;
                    m1 = n1;
                }
                T variance = fmax_(m1 - m0 * m0, (T)0);
                float* o = rad_out + i * 4;
                o[0] = store_rad(st, (float)result.x);
                o[1] = store_rad(st, (float)result.y);
                o[2] = store_rad(st, (float)result.z);
                o[3] = store_rad(st, (float)fmin_(std::sqrt(variance), (T)65000));
                float* mo = mom_out + i * 4;
                mo[0] = (float)m0;
                mo[1] = (float)m1;
                mo[2] = (float)age;
                mo[3] = 0.f;
            }
    }
    // svgf_variance (svgf.wgsl:77-89): temporal + moments[current] -> scratch[0].
    {
        const float* in = st.temporal.data();
        const float* mom = st.moments[current].data();
        float* out = st.scratch[0].data();
#pragma omp parallel for schedule(dynamic, 4) num_threads(st.threads)
        for (int32_t y = (int32_t)st.row0; y < (int32_t)std::min((uint32_t)H, st.row1); y++)
            for (int32_t x = 0; x < W; x++) {
                size_t i = sv.idx(x, y);
                T age = (T)mom[i * 4 + 2];
                T sigma = (T)in[i * 4 + 3];
                if (age < (T)4 && (T)g.depth[i] < (T)1) {
                    T s0 = 0, s1 = 0, total = 0;
                    typename Svgf<T>::Guide a = sv.guide(x, y);
                    for (int32_t yy = -3; yy <= 3; yy++)
                        for (int32_t xx = -3; xx <= 3; xx++) {
                            int32_t qx = x + xx, qy = y + yy;
                            T w = sv.geometry_weight(a, qx, qy, (T)1);
                            if (w <= (T)0) continue;
                            size_t q = sv.idx(qx, qy);
                            s0 += (T)mom[q * 4] * w;
                            s1 += (T)mom[q * 4 + 1] * w;
                            total += w;
                        }
                    T dn = fmax_(total, (T).00001);
                    s0 /= dn;
                    s1 /= dn;
                    sigma = std::sqrt(fmax_(s1 - s0 * s0, (T)0) * (T)4 / fmax_(age, (T)1));
                }
                float* o = out + i * 4;
                o[0] = in[i * 4];
                o[1] = in[i * 4 + 1];
                o[2] = in[i * 4 + 2];
                o[3] = store_rad(st, (float)fmin_(sigma, (T)65000));
            }
    }
    // svgf_atrous x iterations (svgf.wgsl:90-110), ping-pong scratch; the
    // first output also becomes feedback[current] (src/svgf.rs:237-253).
    auto kernel = [](int32_t x) -> T {
        if (x == 0) return (T)1;
        if (x == 1 || x == -1) return (T)2 / (T)3;
        return (T)1 / (T)6;
    };
    for (uint32_t it = 0; it < iterations; it++) {
        const float* in = st.scratch[it % 2].data();
        float* out = st.scratch[1 - it % 2].data();
        int32_t step = (int32_t)(1u << it);
#pragma omp parallel for schedule(dynamic, 4) num_threads(st.threads)
        for (int32_t y = (int32_t)st.row0; y < (int32_t)std::min((uint32_t)H, st.row1); y++)
            for (int32_t x = 0; x < W; x++) {
                size_t i = sv.idx(x, y);
                float* o = out + i * 4;
                if ((T)g.depth[i] >= (T)1) {
                    o[0] = in[i * 4];
                    o[1] = in[i * 4 + 1];
                    o[2] = in[i * 4 + 2];
                    o[3] = in[i * 4 + 3];
                    continue;
                }
                V3<T> c = rgb(in, i);
                T variance = 0, guide_weight = 0;
                typename Svgf<T>::Guide a = sv.guide(x, y);
                for (int32_t yy = -1; yy <= 1; yy++)
                    for (int32_t xx = -1; xx <= 1; xx++) {
                        int32_t qx = std::min(std::max(x + xx, 0), W - 1);
                        int32_t qy = std::min(std::max(y + yy, 0), H - 1);
                        T w = (xx == 0 ? (T)2 : (T)1) * (yy == 0 ? (T)2 : (T)1);
                        T s = (T)in[sv.idx(qx, qy) * 4 + 3];
                        variance += s * s * w;
                        guide_weight += w;
                    }
                T phi = (T)4 * std::sqrt(variance / fmax_(guide_weight, (T).00001)) + (T).0001;
                V3<T> sum = v3<T>(0, 0, 0);
                T total = 0, v = 0;
                T lc = Svgf<T>::lum(c);
                for (int32_t yy = -2; yy <= 2; yy++)
                    for (int32_t xx = -2; xx <= 2; xx++) {
                        int32_t qx = x + xx * step, qy = y + yy * step;
                        T geom = sv.geometry_weight(a, qx, qy, (T)step);
                        if (geom <= (T)0) continue;
                        size_t q = sv.idx(qx, qy);
                        V3<T> smp = rgb(in, q);
                        T sa = (T)in[q * 4 + 3];
                        T w = kernel(xx) * kernel(yy) * geom *
                              std::exp(-std::fabs(Svgf<T>::lum(smp) - lc) / phi);
                        sum = sum + smp * w;
                        v += sa * sa * w * w;
                        total += w;
                    }
                T dn = fmax_(total, (T).00001);
                o[0] = store_rad(st, (float)(sum.x / dn));
                o[1] = store_rad(st, (float)(sum.y / dn));
                o[2] = store_rad(st, (float)(sum.z / dn));
                o[3] = store_rad(st, (float)fmin_(std::sqrt(v) / dn, (T)65000));
            }
        if (it == 0) st.feedback[current] = st.scratch[1];
    }
    st.histories[current] = st.scratch[iterations % 2];
    (void)P;
}

}  // namespace

// ------------------------------------------------------------------ C API
extern "C" {

typedef struct oracle_scene {
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    const irt_light* lights;
    const float* atlas;
    uint32_t atlas_dims[3];
} oracle_scene;

typedef struct oracle_gbuffer {
    const float* depth;
    const float* normal;
    const float* color;
    const float* params;
    const float* motion;
} oracle_gbuffer;

void* oracle_create(uint32_t w, uint32_t h, uint32_t vpl_count, uint32_t max_history, int precision,
                    int radiance_f16, int threads) {
    State* st = new State();
    st->W = w;
    st->H = h;
    st->vpl_count = vpl_count;
    st->max_history = max_history;
    st->precision = precision;
    st->radiance_f16 = radiance_f16;
    st->threads = threads > 0 ? threads : omp_get_max_threads();
    size_t P = (size_t)w * h;
    for (int d = 0; d < 2; d++)
        for (int k = 0; k < 3; k++) st->res[d][k].assign(P, irt_reservoir{});
    st->archive.assign((size_t)(max_history + 1) * vpl_count, irt_vpl{});
    st->prev_depth.assign(P, 0.f);
    st->prev_normal.assign(P * 4, 0.f);
    st->direct_lighting.assign(P * 4, 0.f);
    st->lighting.assign(P * 4, 0.f);
    for (int k = 0; k < 2; k++) {
        st->moments[k].assign(P * 4, 0.f);
        st->feedback[k].assign(P * 4, 0.f);
        st->scratch[k].assign(P * 4, 0.f);
        st->histories[k].assign(P * 4, 0.f);
    }
    st->temporal.assign(P * 4, 0.f);
    return st;
}

void oracle_destroy(void* s) { delete static_cast<State*>(s); }

static Scene to_scene(const oracle_scene* s) {
    Scene sc;
    sc.objects = s->objects;
    sc.meshes = s->meshes;
    sc.nodes = s->nodes;
    sc.lights = s->lights;
    sc.atlas = s->atlas;
    for (int i = 0; i < 3; i++) sc.dims[i] = s->atlas_dims[i];
    return sc;
}
static GBuffer to_gbuffer(const oracle_gbuffer* g) {
    return GBuffer{g->depth, g->normal, g->color, g->params, g->motion};
}

// Lighting passes first..last of the schedule: -1 = archive copy only is
// folded into pass 0; 0 cand_d, 1 cand_i, 2 temp_d, 3 temp_i, 4 spat_d,
// 5 spat_i, 6 resolve_d, 7 resolve_i.
int oracle_lighting(void* s, const irt_frame* f, const oracle_scene* scene, const oracle_gbuffer* gb,
                    const irt_vpl* cur, const irt_vpl* prev, int first_pass, int last_pass) {
    State* st = static_cast<State*>(s);
    if (f->size[0] != st->W || f->size[1] != st->H || f->counts[1] != st->vpl_count) return -1;
    if (f->counts[3] == 0u) return -1;
    Scene sc = to_scene(scene);
    sc.field_linear = st->field_filter;
    GBuffer g = to_gbuffer(gb);
    if (st->precision == 1)
        lighting_passes<double>(*st, *f, sc, g, cur, prev, first_pass, last_pass);
    else
        lighting_passes<float>(*st, *f, sc, g, cur, prev, first_pass, last_pass);
    return 0;
}

int oracle_svgf(void* s, const irt_frame* f, const oracle_gbuffer* gb, uint32_t iterations) {
    State* st = static_cast<State*>(s);
    GBuffer g = to_gbuffer(gb);
    if (st->precision == 1)
        svgf_passes<double>(*st, *f, g, iterations);
    else
        svgf_passes<float>(*st, *f, g, iterations);
    return 0;
}

// End-of-frame history copy of src/renderer.rs:1951-1960.
void oracle_end_frame(void* s, const oracle_gbuffer* gb) {
    State* st = static_cast<State*>(s);
    size_t P = (size_t)st->W * st->H;
    std::copy(gb->depth, gb->depth + P, st->prev_depth.begin());
    std::copy(gb->normal, gb->normal + P * 4, st->prev_normal.begin());
}

int oracle_frame(void* s, const irt_frame* f, const oracle_scene* scene, const oracle_gbuffer* gb,
                 const irt_vpl* cur, const irt_vpl* prev, uint32_t iterations) {
    int r = oracle_lighting(s, f, scene, gb, cur, prev, 0, 7);
    if (r) return r;
    oracle_svgf(s, f, gb, iterations);
    oracle_end_frame(s, gb);
    return 0;
}

// Buffer access for tests (read and write).  which: 0..5 reservoirs
// (domain*3 + k), 6 archive, 7 prev_depth, 8 prev_normal, 9 direct_lighting,
// 10 lighting, 11/12 moments[0/1], 13/14 feedback[0/1], 15 temporal,
// 16/17 scratch[0/1], 18/19 histories[0/1].
void* oracle_buffer(void* s, int which, uint64_t* bytes) {
    State* st = static_cast<State*>(s);
    auto out = [&](auto& v) -> void* {
        *bytes = (uint64_t)(v.size() * sizeof(v[0]));
        return v.data();
    };
    if (which >= 0 && which < 6) return out(st->res[which / 3][which % 3]);
    switch (which) {
    case 6: return out(st->archive);
    case 7: return out(st->prev_depth);
    case 8: return out(st->prev_normal);
    case 9: return out(st->direct_lighting);
    case 10: return out(st->lighting);
    case 11: return out(st->moments[0]);
    case 12: return out(st->moments[1]);
    case 13: return out(st->feedback[0]);
    case 14: return out(st->feedback[1]);
    case 15: return out(st->temporal);
    case 16: return out(st->scratch[0]);
    case 17: return out(st->scratch[1]);
    case 18: return out(st->histories[0]);
    case 19: return out(st->histories[1]);
    }
    *bytes = 0;
    return nullptr;
}

// Counters of the last lighting call: march steps, BVH nodes visited, box
// and field distance queries, visibility rays, light/VPL evaluations.
void oracle_counters(void* s, uint64_t out[6]) {
    State* st = static_cast<State*>(s);
    out[0] = st->last.march_steps;
    out[1] = st->last.nodes;
    out[2] = st->last.box_queries;
    out[3] = st->last.field_queries;
    out[4] = st->last.rays;
    out[5] = st->last.evals;
}

int oracle_threads(void* s) { return static_cast<State*>(s)->threads; }

// Restricts every pass to rows [row0, row1) — used to time a bounded band of
// a large frame; (0, 0xffffffff) restores the whole image.
void oracle_set_rows(void* s, uint32_t row0, uint32_t row1) {
    State* st = static_cast<State*>(s);
    st->row0 = row0;
    st->row1 = row1;
}

// ---- known-answer hooks (src/math.rs) -----------------------------------
uint16_t oracle_f32_to_f16(float v) { return f32_to_f16_rne(v); }
float oracle_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

// random() sequence of seed(i, salt) at frame index `frame`.
void oracle_random_stream(uint32_t i, uint32_t salt, uint32_t frame, uint32_t n, float* out, uint32_t* states) {
    uint32_t s = i * 1973u + frame * 9277u + salt * 26699u + 89173u;
    for (uint32_t k = 0; k < n; k++) {
        out[k] = Path<float>::random(s);
        if (states) states[k] = s;
    }
}

float oracle_signed_box_distance(const float p[3], const float lo[3], const float hi[3]) {
    return Path<float>::signed_box_distance(ld3<float>(p), ld3<float>(lo), ld3<float>(hi));
}

// add() (common.wgsl:100-106) with the random draw replaced by `u`, the form
// of Reservoir::merge in src/math.rs:14-23.  Returns 1 when selected.
int oracle_res_add_u(irt_reservoir* r, uint32_t id, uint32_t source, float target, float pdf, float weight,
                     uint32_t count, uint32_t age, float u) {
    r->count += count;
    if (weight <= 0.f || weight > 1e30f) return 0;
    r->sum += weight;
    if (u * r->sum < weight) {
        r->id = id;
        r->source = source;
        r->selected_target = target;
        r->pdf = pdf;
        r->age = age;
        return 1;
    }
    return 0;
}

float oracle_normalization(const irt_reservoir* r) {
    return Path<float>::normalization(Path<float>::load(*r));
}

// One penumbra update of the march (sdf.wgsl:72-76).
float oracle_quilez_step(float result, float h, float previous, float t, float k) {
    float y = h * h / (2.f * previous);
    float d = std::sqrt(fmax_(h * h - y * y, 0.f));
    if (t > y) result = fmin_(result, k * d / (t - y));
    return result;
}

// Field sampler of the session's march: 0 point-sampled trilinear
// (common.wgsl:31-38), 1 the reference's filtered variant (weights rounded to
// the nearest 1/256), 2 the filtered variant with truncated weights.
void oracle_set_field_filter(void* s, int filter) { static_cast<State*>(s)->field_filter = filter; }

// sample_field of one mesh at grid-space point q over an f32 atlas: the
// point-sampled form or the filtered variant.
float oracle_sample_field(const irt_mesh* mesh, const float* atlas, const uint32_t dims[3], const float q[3],
                          int linear) {
    Scene sc{};
    sc.atlas = atlas;
    for (int i = 0; i < 3; i++) sc.dims[i] = dims[i];
    sc.field_linear = linear;
    irt_frame f{};
    GBuffer g{};
    Path<float> path(f, sc, g, nullptr, nullptr, nullptr, nullptr);
    return path.sample_field(mesh->field, ld3<float>(q), mesh->field[3]);
}

// mesh_distance (sdf.wgsl:5-33) of one mesh over an f32 atlas.
float oracle_mesh_distance(const irt_mesh* mesh, const float* atlas, const uint32_t dims[3], const float p[3]) {
    Scene sc{};
    sc.atlas = atlas;
    for (int i = 0; i < 3; i++) sc.dims[i] = dims[i];
    irt_frame f{};
    GBuffer g{};
    Path<float> path(f, sc, g, nullptr, nullptr, nullptr, nullptr);
    return path.mesh_distance(ld3<float>(p), *mesh);
}

}  // extern "C"
