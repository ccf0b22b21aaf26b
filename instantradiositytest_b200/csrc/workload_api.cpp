// workload_api.cpp — C-ABI of the synthetic workloads, the CPU G-buffer
// producer and the CPU VPL generator (vpl.wgsl:1-47 with analytic ray casts).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "workload.h"

using namespace irt;

namespace irt {

uint32_t oct_encode_snorm16(float x, float y, float z) {
    float s = std::fabs(x) + std::fabs(y) + std::fabs(z);
    float u = x / s, v = y / s;
    if (z < 0.f) {
        float ou = (1.f - std::fabs(v)) * (u >= 0.f ? 1.f : -1.f);
        float ov = (1.f - std::fabs(u)) * (v >= 0.f ? 1.f : -1.f);
        u = ou;
        v = ov;
    }
    auto q = [](float c) {
        c = std::min(std::max(c, -1.f), 1.f);
        return (uint32_t)(uint16_t)(int16_t)std::lrint(c * 32767.f);
    };
    return q(u) | (q(v) << 16);
}

uint32_t pack_unorm8x4(float r, float g, float b, float a) {
    auto q = [](float c) {
        c = std::min(std::max(c, 0.f), 1.f);
        return (uint32_t)std::lrint(c * 255.f);
    };
    return q(r) | (q(g) << 8) | (q(b) << 16) | (q(a) << 24);
}

}  // namespace irt

namespace {

// ---------------------------------------------------------------- f32 shader math (vpl.wgsl)
struct F3 {
    float x, y, z;
};
inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
inline F3 operator*(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 operator/(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline F3 normalize(F3 a) { return a / std::sqrt(dot(a, a)); }
const float PI = 3.14159265359f;

float random(uint32_t& state) {
    state = state * 747796405u + 2891336453u;
    uint32_t w = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (float)((w >> 22u) ^ w) * (1.0f / 4294967296.0f);
}
float luminance(F3 c) { return c.x * .2126f + c.y * .7152f + c.z * .0722f; }

struct Surf {
    F3 p, n, color;
    float rough, metal;
};

F3 brdf(const Surf& s, F3 wo, F3 wi) {
    float nv = std::max(dot(s.n, wo), .00001f);
    float nl = std::max(dot(s.n, wi), 0.f);
    if (nl <= 0.f) return F3{0, 0, 0};
    F3 h = normalize(wo + wi);
    float nh = std::max(dot(s.n, h), 0.f), vh = std::max(dot(wo, h), 0.f);
    float a = s.rough * s.rough, a2 = a * a;
    float q = nh * nh * (a2 - 1.f) + 1.f;
    float d = a2 / (PI * q * q);
    float g1v = 2.f * nv / (nv + std::sqrt(a2 + (1.f - a2) * nv * nv));
    float g1l = 2.f * nl / (nl + std::sqrt(a2 + (1.f - a2) * nl * nl));
    F3 f0 = F3{.04f, .04f, .04f} * (1.f - s.metal) + s.color * s.metal;
    float p5 = std::pow(1.f - vh, 5.f);
    F3 f = f0 + (F3{1, 1, 1} - f0) * p5;
    F3 diffuse = (F3{1, 1, 1} - f) * (1.f - s.metal) * s.color / PI;
    F3 spec = f * d * g1v * g1l / std::max(4.f * nv * nl, .00001f);
    return diffuse + spec;
}
// basis() of common.wgsl:84: columns t, cross(n, t), n.
void basis(F3 n, F3& t, F3& b) {
    F3 axis = std::fabs(n.z) > .9f ? F3{1, 0, 0} : F3{0, 0, 1};
    t = normalize(cross(axis, n));
    b = cross(n, t);
}
F3 apply_basis(F3 n, F3 v) {
    F3 t, b;
    basis(n, t, b);
    return t * v.x + b * v.y + n * v.z;
}
F3 cosine_direction(F3 n, uint32_t& rng) {
    float u = random(rng);
    float phi = 2.f * PI * random(rng);
    return apply_basis(n, F3{std::sqrt(u) * std::cos(phi), std::sqrt(u) * std::sin(phi), std::sqrt(1.f - u)});
}
// sample_bsdf (common.wgsl:87-97).
void sample_bsdf(const Surf& s, F3 wo, uint32_t& rng, F3& wi, F3& weight) {
    float spec_probability = .25f * (1.f - s.metal) + .9f * s.metal;
    if (random(rng) < spec_probability) {
        float a2 = std::pow(s.rough, 4.f);
        float u = random(rng);
        float cos_theta = std::sqrt((1.f - u) / (1.f + (a2 - 1.f) * u));
        float phi = 2.f * PI * random(rng);
        float st = std::sqrt(1.f - cos_theta * cos_theta);
        F3 h = apply_basis(s.n, F3{st * std::cos(phi), st * std::sin(phi), cos_theta});
        F3 i = -wo;
        wi = i - h * (2.f * dot(h, i));
    } else {
        wi = cosine_direction(s.n, rng);
    }
    float nl = std::max(dot(s.n, wi), 0.f);
    if (nl <= 0.f) {
        weight = F3{0, 0, 0};
        return;
    }
    F3 h = normalize(wo + wi);
    float nh = std::max(dot(s.n, h), 0.f);
    float a2 = std::pow(s.rough, 4.f);
    float q = nh * nh * (a2 - 1.f) + 1.f;
    float pdf_d = nl / PI;
    float pdf_s = a2 * nh / (PI * q * q * std::max(4.f * std::fabs(dot(wo, h)), .00001f));
    float pdf = pdf_d * (1.f - spec_probability) + pdf_s * spec_probability;
    weight = brdf(s, wo, wi) * nl / std::max(pdf, .00001f);
}

}  // namespace

extern "C" {

irt_status irt_workload_preset(int32_t which, irt_workload_spec* s) {
    if (!s) return IRT_E_INVALID;
    std::memset(s, 0, sizeof(*s));
    s->sdf_format = IRT_SDF_F32;
    s->vpl_bounces = 3;
    switch (which) {
    case 0:  // 256x160, 16 frames: 6 walls + 4 boxes + 2 spheres, 64^3, one emitter
        s->seed = 0;
        s->width = 256;
        s->height = 160;
        s->n_boxes = 4;
        s->n_spheres = 2;
        s->room_single_mesh = 0;
        s->sdf_resolution = 64;
        s->n_lights = 1;
        s->radiance_lo = s->radiance_hi = 20.f;
        s->emitter_size_lo = s->emitter_size_hi = 0.5f;
        s->vpl_count = 100;
        s->orbit_deg_per_frame = 0.5f;
        s->dolly_m_per_frame = 0.f;
        return IRT_OK;
    case 1:  // 1920x1200, 64 frames: room + 14 boxes + 9 spheres, 128^3, 8 emitters
    case 2:  // same scene with fp16 SDF storage
        s->seed = 0;
        s->width = 1920;
        s->height = 1200;
        s->n_boxes = 14;
        s->n_spheres = 9;
        s->room_single_mesh = 1;
        s->sdf_resolution = 128;
        s->sdf_format = which == 2 ? IRT_SDF_F16 : IRT_SDF_F32;
        s->n_lights = 8;
        s->radiance_lo = 5.f;
        s->radiance_hi = 40.f;
        s->emitter_size_lo = 0.2f;
        s->emitter_size_hi = 1.f;
        s->vpl_count = 1024;
        s->orbit_deg_per_frame = 1.f;
        s->dolly_m_per_frame = 0.05f;
        return IRT_OK;
    }
    return IRT_E_INVALID;
}

void irt_workload_destroy(irt_workload* wl) {
    if (!wl) return;
    if (wl->w.release_device) wl->w.release_device(wl->w);
    delete wl;
}

irt_status irt_workload_create(const irt_workload_spec* spec, irt_workload** out) {
    if (!spec || !out) return IRT_E_INVALID;
    if (spec->width == 0 || spec->height == 0 || spec->width > 8192 || spec->height > 8192) return IRT_E_INVALID;
    if (spec->sdf_resolution < 4 || spec->sdf_resolution > 256) return IRT_E_INVALID;
    if (spec->vpl_count == 0 || spec->vpl_bounces == 0) return IRT_E_INVALID;
    irt_workload* wl = new (std::nothrow) irt_workload();
    if (!wl) return IRT_E_NOMEM;
    wl->w.spec = *spec;
    if (!wl->w.build()) {
        delete wl;
        return IRT_E_INVALID;
    }
    *out = wl;
    return IRT_OK;
}

uint32_t irt_workload_mesh_count(const irt_workload* wl) { return (uint32_t)wl->w.meshes.size(); }
uint32_t irt_workload_object_count(const irt_workload* wl) { return (uint32_t)wl->w.objs.size(); }
uint32_t irt_workload_light_count(const irt_workload* wl) { return (uint32_t)wl->w.lights.size(); }
const irt_mesh* irt_workload_meshes(const irt_workload* wl) { return wl->w.meshes.data(); }
int32_t irt_workload_sdf_format(const irt_workload* wl) { return wl->w.spec.sdf_format; }
const void* irt_workload_atlas(const irt_workload* wl, uint32_t dims_out[3]) {
    for (int i = 0; i < 3; i++) dims_out[i] = wl->w.atlas_dims[i];
    if (wl->w.spec.sdf_format == IRT_SDF_F16) return wl->w.atlas16.data();
    return wl->w.atlas32.data();
}
void irt_workload_settings(const irt_workload* wl, irt_settings* out) { wl->w.settings(out); }

irt_status irt_workload_frame(irt_workload* wl, uint32_t index, uint32_t debug, irt_frame* frame,
                              irt_object* objects, irt_node* nodes, irt_light* lights) {
    if (!wl || !frame || !objects || !nodes || !lights) return IRT_E_INVALID;
    wl->w.frame_data(index, debug, frame, objects, nodes, lights);
    return IRT_OK;
}

// CPU G-buffer producer: one analytic primary ray per pixel centre.
irt_status irt_workload_gbuffer_cpu(const irt_workload* wl, const irt_frame* f, const irt_object* objects,
                                    int32_t format, float* depth, void* normal, void* color, void* params,
                                    void* motion) {
    (void)objects;
    if (!wl || !f || !depth || !normal || !color || !params || !motion) return IRT_E_INVALID;
    if (format < IRT_GBUFFER_F32 || format > IRT_GBUFFER_PACKED) return IRT_E_INVALID;
    const Workload& w = wl->w;
    const uint32_t W = f->size[0], H = f->size[1];
    M4 vp = from_f32(f->vp), inv_vp = from_f32(f->inv_vp), prev_vp = from_f32(f->previous_vp);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t yy = 0; yy < (int64_t)H; yy++) {
        uint32_t y = (uint32_t)yy;
        for (uint32_t x = 0; x < W; x++) {
            size_t i = (size_t)y * W + x;
            double u = ((double)x + 0.5) / W, v = ((double)y + 0.5) / H;
            double nx = u * 2 - 1, ny = 1 - v * 2;
            double pn[4], pf[4];
            transform(inv_vp, nx, ny, 0.0, 1.0, pn);
            transform(inv_vp, nx, ny, 1.0, 1.0, pf);
            double o[3] = {pn[0] / pn[3], pn[1] / pn[3], pn[2] / pn[3]};
            double e[3] = {pf[0] / pf[3], pf[1] / pf[3], pf[2] / pf[3]};
            double d[3] = {e[0] - o[0], e[1] - o[1], e[2] - o[2]};
            double t, n[3];
            uint32_t obj = 0;
            float dep = 1.f, nrm[3] = {0, 0, 0}, col[3] = {0, 0, 0}, par[2] = {0, 0}, mot[2] = {0, 0};
            bool hit = w.cast(o, d, 0.0, 1.0, t, n, obj, true);
            if (hit) {
                double p[3] = {o[0] + d[0] * t, o[1] + d[1] * t, o[2] + d[2] * t};
                double c[4], pc[4];
                transform(vp, p[0], p[1], p[2], 1.0, c);
                transform(prev_vp, p[0], p[1], p[2], 1.0, pc);
                dep = (float)(c[2] / c[3]);
                if (dep >= 1.f) dep = std::nextafter(1.f, 0.f);
                for (int k = 0; k < 3; k++) nrm[k] = (float)n[k];
                const irt_material& m = w.materials[w.objs[obj].material];
                for (int k = 0; k < 3; k++) col[k] = m.color[k];
                par[0] = std::min(std::max(m.params[0], .045f), 1.f);
                par[1] = std::min(std::max(m.params[1], 0.f), 1.f);
                mot[0] = (float)((c[0] / c[3] - pc[0] / pc[3]) * 0.5);
                mot[1] = (float)((c[1] / c[3] - pc[1] / pc[3]) * -0.5);
            }
            depth[i] = dep;
            if (format == IRT_GBUFFER_F32) {
                float* nn = (float*)normal + i * 4;
                float* cc = (float*)color + i * 4;
                nn[0] = nrm[0];
                nn[1] = nrm[1];
                nn[2] = nrm[2];
                nn[3] = hit ? 1.f : 0.f;
                cc[0] = col[0];
                cc[1] = col[1];
                cc[2] = col[2];
                cc[3] = hit ? 1.f : 0.f;
                ((float*)params)[i * 2] = par[0];
                ((float*)params)[i * 2 + 1] = par[1];
                ((float*)motion)[i * 2] = mot[0];
                ((float*)motion)[i * 2 + 1] = mot[1];
            } else if (format == IRT_GBUFFER_F16) {
                uint16_t* nn = (uint16_t*)normal + i * 4;
                uint16_t* cc = (uint16_t*)color + i * 4;
                for (int k = 0; k < 3; k++) {
                    nn[k] = f16_bits_rne(nrm[k]);
                    cc[k] = f16_bits_rne(col[k]);
                }
                nn[3] = f16_bits_rne(hit ? 1.f : 0.f);
                cc[3] = f16_bits_rne(hit ? 1.f : 0.f);
                ((uint16_t*)params)[i * 2] = f16_bits_rne(par[0]);
                ((uint16_t*)params)[i * 2 + 1] = f16_bits_rne(par[1]);
                ((uint16_t*)motion)[i * 2] = f16_bits_rne(mot[0]);
                ((uint16_t*)motion)[i * 2 + 1] = f16_bits_rne(mot[1]);
            } else {
                ((uint32_t*)normal)[i] = hit ? oct_encode_snorm16(nrm[0], nrm[1], nrm[2]) : 0u;
                ((uint32_t*)color)[i] = pack_unorm8x4(col[0], col[1], col[2], hit ? 1.f : 0.f);
                ((uint16_t*)params)[i * 2] = f16_bits_rne(par[0]);
                ((uint16_t*)params)[i * 2 + 1] = f16_bits_rne(par[1]);
                ((uint16_t*)motion)[i * 2] = f16_bits_rne(mot[0]);
                ((uint16_t*)motion)[i * 2 + 1] = f16_bits_rne(mot[1]);
            }
        }
    }
    return IRT_OK;
}

// CPU VPL generator: vpl.wgsl:1-47 (light-path tracing with Russian
// roulette; the record keeps the path's terminal vertex) with analytic ray
// casts for the hardware ray query (t in [0.0005, 10000]).
irt_status irt_workload_vpls_cpu(const irt_workload* wl, const irt_frame* f, const irt_object* objects,
                                 const irt_light* lights, irt_vpl* out) {
    (void)objects;
    if (!wl || !f || !lights || !out) return IRT_E_INVALID;
    const Workload& w = wl->w;
    const uint32_t n = f->counts[1];
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ii = 0; ii < (int64_t)n; ii++) {
        uint32_t id = (uint32_t)ii;
        uint32_t rng = id * 1973u + f->size[2] * 9277u + 7u * 26699u + 89173u;
        irt_vpl v{};
        if (f->counts[0] == 0u) {
            out[id] = v;
            continue;
        }
        uint32_t light_id = std::min((uint32_t)(random(rng) * (float)f->counts[0]), f->counts[0] - 1u);
        const irt_light& l = lights[light_id];
        F3 origin{l.position_strength[0], l.position_strength[1], l.position_strength[2]};
        F3 direction;
        float omega = 4.f * PI;
        if (l.color_type[3] > .5f) {
            float ca = std::cos(l.direction_angle[3] * .5f);
            omega = 2.f * PI * (1.f - ca);
            float u = random(rng);
            float z = ca * (1.f - u) + 1.f * u;
            float phi = 2.f * PI * random(rng);
            F3 axis = normalize(F3{l.direction_angle[0], l.direction_angle[1], l.direction_angle[2]});
            float s = std::sqrt(1.f - z * z);
            direction = apply_basis(axis, F3{s * std::cos(phi), s * std::sin(phi), z});
        } else {
            float z = 2.f * random(rng) - 1.f;
            float phi = 2.f * PI * random(rng);
            float s = std::sqrt(1.f - z * z);
            direction = F3{s * std::cos(phi), s * std::sin(phi), z};
        }
        F3 color{l.color_type[0], l.color_type[1], l.color_type[2]};
        F3 source_flux = color * l.position_strength[3] * omega * (float)f->counts[0];
        F3 throughput{1, 1, 1};
        for (uint32_t bounce = 0; bounce < f->counts[2]; bounce++) {
            double o[3] = {origin.x, origin.y, origin.z}, d[3] = {direction.x, direction.y, direction.z};
            double t, nn[3];
            uint32_t obj = 0;
            if (!w.cast(o, d, 0.0005, 10000.0, t, nn, obj)) {
                v.flux[0] = v.flux[1] = v.flux[2] = v.flux[3] = 0.f;
                break;
            }
            const irt_material& m = w.materials[w.objs[obj].material];
            Surf s;
            s.color = F3{m.color[0], m.color[1], m.color[2]};
            s.rough = std::min(std::max(m.params[0], .045f), 1.f);
            s.metal = std::min(std::max(m.params[1], 0.f), 1.f);
            s.n = normalize(F3{(float)nn[0], (float)nn[1], (float)nn[2]});
            s.p = origin + direction * (float)t;
            F3 wo = -direction;
            if (dot(s.n, wo) <= 0.f) {
                v.flux[0] = v.flux[1] = v.flux[2] = v.flux[3] = 0.f;
                break;
            }
            v.position[0] = s.p.x;
            v.position[1] = s.p.y;
            v.position[2] = s.p.z;
            v.position[3] = 1.f;
            v.normal[0] = s.n.x;
            v.normal[1] = s.n.y;
            v.normal[2] = s.n.z;
            v.normal[3] = 0.f;
            F3 wi, weight;
            sample_bsdf(s, wo, rng, wi, weight);
            F3 reflected = throughput * weight;
            F3 flux = source_flux * reflected / (float)f->counts[1];
            v.flux[0] = flux.x;
            v.flux[1] = flux.y;
            v.flux[2] = flux.z;
            v.flux[3] = 0.f;
            if (bounce + 1u >= f->counts[2]) break;
            float survive = std::min(std::max(std::max(reflected.x, std::max(reflected.y, reflected.z)), f->rr[0]), f->rr[1]);
            if (random(rng) > survive) break;
            if (luminance(weight) <= 0.f) break;
            throughput = reflected / survive;
            origin = s.p + s.n * .001f;
            direction = wi;
        }
        out[id] = v;
    }
    return IRT_OK;
}

}  // extern "C"
