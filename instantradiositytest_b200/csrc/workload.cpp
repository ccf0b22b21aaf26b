// workload.cpp — seeded procedural rooms (the synthetic workloads the lighting
// path is measured on) and the host-side input producers:
//   * per-frame packing of the Frame uniform, objects, BVH and lights as
//     Renderer::encode does (src/renderer.rs:1675-1782);
//   * a CPU G-buffer producer casting analytic primary rays (stands in for the
//     gbuffer.wgsl raster: depth in [0,1] DirectX convention, normal, colour,
//     roughness/metal, motion = (ndc - previous ndc) * (.5, -.5));
//   * a CPU VPL generator following vpl.wgsl:1-47 with analytic ray casts in
//     place of the hardware ray query.
// Scenes are Z-up rooms: a 10 m cube centred at the origin whose six walls
// are closed 0.2 m slabs, axis-aligned boxes resting on the floor, spheres,
// and quad emitters mapped to wide spot lights on the ceiling.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "host_math.h"
#include "workload.h"

using namespace irt;

namespace {

// splitmix64 (Steele, Lea, Flood 2014).
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double lo, double hi) { return lo + (hi - lo) * uniform(); }
};

const double kRoomHalf = 5.0;
const double kWallHalf = 0.1;
const double kFloorTop = -kRoomHalf + kWallHalf;  // -4.9
const double kCameraHeight = 1.6;

void box_mesh(const double lo[3], const double hi[3], std::vector<irt_vertex>& v, std::vector<uint32_t>& idx) {
    uint32_t base = (uint32_t)v.size();
    for (int i = 0; i < 8; i++) {
        irt_vertex vx{};
        vx.position[0] = (float)((i & 1) ? hi[0] : lo[0]);
        vx.position[1] = (float)((i & 2) ? hi[1] : lo[1]);
        vx.position[2] = (float)((i & 4) ? hi[2] : lo[2]);
        vx.position[3] = 1.f;
        v.push_back(vx);
    }
    // Two triangles per side, each pair sharing a face diagonal.
    static const uint32_t tri[36] = {0, 2, 6, 0, 6, 4, 1, 5, 7, 1, 7, 3, 0, 4, 5, 0, 5, 1,
                                     2, 3, 7, 2, 7, 6, 0, 1, 3, 0, 3, 2, 4, 6, 7, 4, 7, 5};
    for (uint32_t t : tri) idx.push_back(base + t);
}

void sphere_mesh(double r, std::vector<irt_vertex>& v, std::vector<uint32_t>& idx) {
    const int stacks = 16, slices = 32;
    for (int i = 0; i <= stacks; i++) {
        double th = M_PI * i / stacks;
        for (int j = 0; j < slices; j++) {
            double ph = 2 * M_PI * j / slices;
            irt_vertex vx{};
            vx.position[0] = (float)(r * std::sin(th) * std::cos(ph));
            vx.position[1] = (float)(r * std::sin(th) * std::sin(ph));
            vx.position[2] = (float)(r * std::cos(th));
            vx.position[3] = 1.f;
            v.push_back(vx);
        }
    }
    for (int i = 0; i < stacks; i++)
        for (int j = 0; j < slices; j++) {
            uint32_t a = i * slices + j, b = i * slices + (j + 1) % slices;
            uint32_t c = (i + 1) * slices + j, d = (i + 1) * slices + (j + 1) % slices;
            idx.insert(idx.end(), {a, c, b, b, c, d});
        }
}

double box_sdf(const double p[3], const double lo[3], const double hi[3]) {
    double d[3], outside = 0, inside = -1e300;
    for (int a = 0; a < 3; a++) {
        d[a] = std::max(lo[a] - p[a], p[a] - hi[a]);
        outside += std::max(d[a], 0.0) * std::max(d[a], 0.0);
        inside = std::max(inside, d[a]);
    }
    return std::sqrt(outside) + std::min(inside, 0.0);
}

// Ray / AABB slab test; returns entry t and the outward normal of the entry face.
bool ray_box(const double o[3], const double d[3], const double lo[3], const double hi[3], double tmin,
             double tmax, double& t, double n[3]) {
    double t0 = tmin, t1 = tmax;
    int axis = -1;
    double sign = 0;
    for (int a = 0; a < 3; a++) {
        double inv = 1.0 / d[a];
        double ta = (lo[a] - o[a]) * inv, tb = (hi[a] - o[a]) * inv;
        double s = -1;
        if (ta > tb) {
            std::swap(ta, tb);
            s = 1;
        }
        if (ta > t0) {
            t0 = ta;
            axis = a;
            sign = s;
        }
        t1 = std::min(t1, tb);
        if (t0 > t1) return false;
    }
    if (axis < 0) return false;  // origin inside the box
    t = t0;
    n[0] = n[1] = n[2] = 0;
    n[axis] = sign;
    return true;
}

bool ray_sphere(const double o[3], const double d[3], double r, double tmin, double tmax, double& t, double n[3]) {
    double b = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
    double a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double c = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - r * r;
    double disc = b * b - a * c;
    if (disc < 0) return false;
    double s = std::sqrt(disc);
    double t0 = (-b - s) / a;
    if (t0 < tmin || t0 > tmax) return false;  // only front entries count
    t = t0;
    for (int k = 0; k < 3; k++) n[k] = (o[k] + d[k] * t) / r;
    return true;
}

}  // namespace

namespace irt {

// Local-space intersection of one object's primitive set.
bool Workload::intersect_object(uint32_t oi, const double ow[3], const double dw[3], double tmin, double tmax,
                                double& t, double nw[3], bool cull) const {
    const Obj& ob = objs[oi];
    const MeshDesc& md = mesh_desc[ob.mesh];
    double o[4], d[4];
    transform(ob.inv_model, ow[0], ow[1], ow[2], 1.0, o);
    transform(ob.inv_model, dw[0], dw[1], dw[2], 0.0, d);
    bool hit = false;
    double nl[3];
    if (md.triangles) hit = cast_tri_bvh(md.bvh, o, d, tmin, tmax, cull, t, nl);
    for (const Part& p : md.parts) {
        double tt, nn[3];
        bool h = p.sphere ? ray_sphere(o, d, p.radius, tmin, tmax, tt, nn)
                          : ray_box(o, d, p.lo, p.hi, tmin, tmax, tt, nn);
        if (h && tt < tmax) {
            tmax = tt;
            t = tt;
            nl[0] = nn[0];
            nl[1] = nn[1];
            nl[2] = nn[2];
            hit = true;
        }
    }
    if (!hit) return false;
    double w[4];
    transform(ob.model, nl[0], nl[1], nl[2], 0.0, w);
    D3 nn = normalize(D3{w[0], w[1], w[2]});
    nw[0] = nn.x;
    nw[1] = nn.y;
    nw[2] = nn.z;
    return true;
}

bool Workload::cast(const double o[3], const double d[3], double tmin, double tmax, double& t, double n[3],
                    uint32_t& object, bool cull) const {
    bool hit = false;
    for (uint32_t i = 0; i < objs.size(); i++) {
        double tt, nn[3];
        if (intersect_object(i, o, d, tmin, tmax, tt, nn, cull)) {
            tmax = tt;
            t = tt;
            n[0] = nn[0];
            n[1] = nn[1];
            n[2] = nn[2];
            object = i;
            hit = true;
        }
    }
    return hit;
}

void Workload::camera_at(uint32_t frame, double eye[3], double target[3]) const {
    if (loaded) {
        // Fixed camera: eye at its position, looking down its local -z.
        double q[4] = {cam_q[0], cam_q[1], cam_q[2], cam_q[3]};
        M4 r = scale_rotation_translation(1.0, q, D3{0, 0, 0});
        double fwd[4];
        transform(r, 0, 0, -1, 0, fwd);
        for (int a = 0; a < 3; a++) {
            eye[a] = cam_eye[a];
            target[a] = cam_eye[a] + fwd[a];
        }
        return;
    }
    // Orbit and dolly follow a triangle wave of period 2*kPathFrames so the
    // camera sweeps a fixed sector however many frames are rendered.
    double period = 2.0 * path_frames;
    double ph = std::fmod((double)frame, period);
    double k = ph <= path_frames ? ph : period - ph;
    double angle = (spec.orbit_deg_per_frame * k) * M_PI / 180.0 + angle0;
    double radius = 4.0 - spec.dolly_m_per_frame * k;
    double z = kFloorTop + kCameraHeight;
    eye[0] = radius * std::cos(angle);
    eye[1] = radius * std::sin(angle);
    eye[2] = z;
    target[0] = 0;
    target[1] = 0;
    target[2] = kFloorTop + 0.9;
}

M4 Workload::view_projection(uint32_t frame) const {
    if (loaded) {
        // Camera::matrix (src/scene.rs:119-128): perspective (right-handed,
        // depth 0..1) times the inverse of the camera's rotation-translation.
        double q[4] = {cam_q[0], cam_q[1], cam_q[2], cam_q[3]};
        M4 pose = scale_rotation_translation(1.0, q, D3{cam_eye[0], cam_eye[1], cam_eye[2]});
        M4 proj = perspective_rh_zo(cam_fov, (double)spec.width / (double)spec.height, cam_near, cam_far);
        return mul(proj, inverse(pose));
    }
    double eye[3], target[3];
    camera_at(frame, eye, target);
    M4 view = look_at_rh(D3{eye[0], eye[1], eye[2]}, D3{target[0], target[1], target[2]}, D3{0, 0, 1});
    M4 proj = perspective_rh_zo(0.9, (double)spec.width / (double)spec.height, 0.1, 1000.0);
    return mul(proj, view);
}

bool Workload::build() {
    SplitMix rng{spec.seed * 0x2545F4914F6CDD1Dull + 0x1234567ull};
    path_frames = 64;
    angle0 = 0.0;
    auto add_mesh = [&](MeshDesc md) {
        mesh_desc.push_back(md);
        return (uint32_t)mesh_desc.size() - 1;
    };
    auto add_object = [&](uint32_t mesh, D3 pos, double scale, double yaw, const float color[3]) {
        Obj o;
        o.mesh = mesh;
        o.material = (uint32_t)materials.size();
        double q[4] = {0, 0, std::sin(yaw * 0.5), std::cos(yaw * 0.5)};
        o.model = scale_rotation_translation(scale, q, pos);
        o.inv_model = inverse(o.model);
        objs.push_back(o);
        irt_material m{};
        m.color[0] = color[0];
        m.color[1] = color[1];
        m.color[2] = color[2];
        m.color[3] = 1.f;
        m.params[0] = 1.f;  // roughness (Lambertian room: rough 1, metal 0)
        m.params[1] = 0.f;
        m.params[2] = 1.f;
        m.params[3] = 0.f;
        for (int k = 0; k < 4; k++) m.textures[k] = -1;
        materials.push_back(m);
    };
    auto albedo = [&](float c[3]) {
        for (int k = 0; k < 3; k++) c[k] = (float)rng.uniform(0.2, 0.9);
    };
    // Walls: six slabs of thickness 0.2 m centred on the cube faces.
    std::vector<Part> slabs;
    for (int axis = 0; axis < 3; axis++)
        for (int side = 0; side < 2; side++) {
            Part p{};
            for (int a = 0; a < 3; a++) {
                p.lo[a] = -kRoomHalf - kWallHalf;
                p.hi[a] = kRoomHalf + kWallHalf;
            }
            double c = side ? kRoomHalf : -kRoomHalf;
            p.lo[axis] = c - kWallHalf;
            p.hi[axis] = c + kWallHalf;
            slabs.push_back(p);
        }
    if (spec.room_single_mesh) {
        MeshDesc md;
        md.parts = slabs;
        float c[3];
        albedo(c);
        add_object(add_mesh(md), D3{0, 0, 0}, 1.0, 0.0, c);
    } else {
        for (const Part& s : slabs) {
            // Each wall is its own box mesh centred at the origin of its object.
            MeshDesc md;
            Part p = s;
            double ctr[3];
            for (int a = 0; a < 3; a++) {
                ctr[a] = 0.5 * (s.lo[a] + s.hi[a]);
                p.lo[a] = s.lo[a] - ctr[a];
                p.hi[a] = s.hi[a] - ctr[a];
            }
            md.parts.push_back(p);
            float c[3];
            albedo(c);
            add_object(add_mesh(md), D3{ctr[0], ctr[1], ctr[2]}, 1.0, 0.0, c);
        }
    }
    // Camera path samples for placement rejection.
    std::vector<D3> path;
    for (uint32_t f = 0; f <= 2 * path_frames; f++) {
        double e[3], t[3];
        camera_at(f, e, t);
        path.push_back(D3{e[0], e[1], 0});
    }
    struct Placed {
        double x, y, rho;
    };
    std::vector<Placed> placed;
    auto free_spot = [&](double x, double y, double rho, bool strict) {
        for (const D3& c : path)
            if (std::hypot(x - c.x, y - c.y) < rho + 0.45) return false;
        if (strict)
            for (const Placed& p : placed)
                if (std::hypot(x - p.x, y - p.y) < rho + p.rho + 0.05) return false;
        return true;
    };
    auto place = [&](double rho, double& x, double& y) {
        double lim = kRoomHalf - kWallHalf - rho - 0.02;
        for (int attempt = 0; attempt < 4000; attempt++) {
            x = rng.uniform(-lim, lim);
            y = rng.uniform(-lim, lim);
            if (free_spot(x, y, rho, attempt < 2000)) {
                placed.push_back(Placed{x, y, rho});
                return true;
            }
        }
        return false;
    };
    for (uint32_t b = 0; b < spec.n_boxes; b++) {
        double h[3];
        for (int a = 0; a < 3; a++) h[a] = 0.5 * rng.uniform(0.5, 2.0);
        double x, y;
        if (!place(std::hypot(h[0], h[1]), x, y)) return false;
        MeshDesc md;
        Part p{};
        for (int a = 0; a < 3; a++) {
            p.lo[a] = -h[a];
            p.hi[a] = h[a];
        }
        md.parts.push_back(p);
        float c[3];
        albedo(c);
        add_object(add_mesh(md), D3{x, y, kFloorTop + h[2]}, 1.0, 0.0, c);
    }
    for (uint32_t s = 0; s < spec.n_spheres; s++) {
        double r = rng.uniform(0.3, 1.0);
        double scale = rng.uniform(0.8, 1.25);
        double yaw = rng.uniform(0.0, 2 * M_PI);
        double lift = rng.uniform(0.0, 1.5);
        double x, y;
        if (!place(r, x, y)) return false;
        MeshDesc md;
        Part p{};
        p.sphere = true;
        p.radius = r / scale;
        md.parts.push_back(p);
        float c[3];
        albedo(c);
        add_object(add_mesh(md), D3{x, y, kFloorTop + r + lift}, scale, yaw, c);
    }
    // Emitters: quads of side `size` and radiance L on the ceiling, as spot
    // lights aimed down with angle 0.999*pi and strength L * size^2.
    for (uint32_t l = 0; l < spec.n_lights; l++) {
        double L = spec.n_lights == 1 ? spec.radiance_lo : rng.uniform(spec.radiance_lo, spec.radiance_hi);
        double size = spec.n_lights == 1 ? spec.emitter_size_lo : rng.uniform(spec.emitter_size_lo, spec.emitter_size_hi);
        double x = spec.n_lights == 1 ? 0.0 : rng.uniform(-4.0, 4.0);
        double y = spec.n_lights == 1 ? 0.0 : rng.uniform(-4.0, 4.0);
        irt_light li{};
        li.position_strength[0] = (float)x;
        li.position_strength[1] = (float)y;
        // 0.05 m below the ceiling when the walls are certified boxes (exact
        // distances).  A room that is one field mesh has the field bias
        // voxel diagonal * (0.5 + 1/128) (~0.07 m at 128^3 over the room)
        // plus the march clearance (0.65 voxel) around its surface, so a
        // light closer than ~0.13 m would sit inside it and every shadow ray
        // to it would end occluded: those emitters hang 0.5 m below.
        li.position_strength[2] = (float)(kRoomHalf - kWallHalf - (spec.room_single_mesh ? 0.5 : 0.05));
        li.position_strength[3] = (float)(L * size * size);
        li.direction_angle[0] = 0.f;
        li.direction_angle[1] = 0.f;
        li.direction_angle[2] = -1.f;
        li.direction_angle[3] = (float)(0.999 * M_PI);
        li.color_type[0] = li.color_type[1] = li.color_type[2] = 1.f;
        li.color_type[3] = 1.f;
        lights.push_back(li);
    }
    // Mesh geometry, SDF grids, metadata and atlas.
    uint32_t res = spec.sdf_resolution;
    uint32_t count = (uint32_t)mesh_desc.size();
    irt_atlas_layout(count, res, atlas_grid, atlas_dims);
    size_t texels = (size_t)atlas_dims[0] * atlas_dims[1] * atlas_dims[2];
    if (spec.sdf_format == IRT_SDF_F16)
        atlas16.assign(texels, 0);
    else
        atlas32.assign(texels, 0.f);
    meshes.resize(count);
    for (uint32_t m = 0; m < count; m++) {
        MeshDesc& md = mesh_desc[m];
        for (const Part& p : md.parts) {
            if (p.sphere)
                sphere_mesh(p.radius, md.vertices, md.indices);
            else
                box_mesh(p.lo, p.hi, md.vertices, md.indices);
        }
    }
    // Meshes are independent (each writes its own atlas tile): one thread
    // per mesh samples its grid, derives its metadata and fills its tile.
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t mi = 0; mi < (int64_t)count; mi++) {
        const uint32_t m = (uint32_t)mi;
        MeshDesc& md = mesh_desc[m];
        md.resolution = res;
        // Exporter SDF conventions (tools/export_scene.py:136-152): padding of
        // two voxels of the vertex-box diagonal, bias of -extent * 2e-6.
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (const irt_vertex& v : md.vertices)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], (double)v.position[a]);
                hi[a] = std::max(hi[a], (double)v.position[a]);
            }
        double diag = std::sqrt((hi[0] - lo[0]) * (hi[0] - lo[0]) + (hi[1] - lo[1]) * (hi[1] - lo[1]) +
                                (hi[2] - lo[2]) * (hi[2] - lo[2]));
        double pad = diag / (res - 1) * 2;
        for (int a = 0; a < 3; a++) {
            md.sdf_lo[a] = (float)(lo[a] - pad);
            md.sdf_hi[a] = (float)(hi[a] + pad);
        }
        double ext = std::sqrt(std::pow(md.sdf_hi[0] - md.sdf_lo[0], 2) + std::pow(md.sdf_hi[1] - md.sdf_lo[1], 2) +
                               std::pow(md.sdf_hi[2] - md.sdf_lo[2], 2));
        std::vector<float> smp((size_t)res * res * res);
        for (uint32_t z = 0; z < res; z++)
            for (uint32_t y = 0; y < res; y++)
                for (uint32_t x = 0; x < res; x++) {
                    double p[3];
                    uint32_t c[3] = {x, y, z};
                    for (int a = 0; a < 3; a++)
                        p[a] = md.sdf_lo[a] + ((double)md.sdf_hi[a] - md.sdf_lo[a]) * c[a] / (res - 1);
                    double d = 1e300;
                    for (const Part& part : md.parts) {
                        double v;
                        if (part.sphere)
                            v = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]) - part.radius;
                        else
                            v = box_sdf(p, part.lo, part.hi);
                        d = std::min(d, v);
                    }
                    smp[((size_t)z * res + y) * res + x] = (float)(d - ext * 2e-6);
                }
        uint32_t origin[3] = {(m % atlas_grid[0]) * res, ((m / atlas_grid[0]) % atlas_grid[1]) * res,
                              (m / (atlas_grid[0] * atlas_grid[1])) * res};
        irt_mesh_metadata(md.vertices.data(), (uint32_t)md.vertices.size(), md.indices.data(),
                          (uint32_t)md.indices.size(), smp.data(), res, md.sdf_lo, md.sdf_hi, origin, &meshes[m]);
        store_field(m, smp.data(), res, origin);
    }
    // Static scene: previous transforms equal the current ones.
    return true;
}

void Workload::store_field(uint32_t m, const float* smp, uint32_t res, const uint32_t origin[3]) {
    float scale = 1.f;
    if (spec.sdf_format == IRT_SDF_F16) {
        scale = meshes[m].grid[3];
        meshes[m].lo[3] = scale;
    }
    for (uint32_t z = 0; z < res; z++)
        for (uint32_t y = 0; y < res; y++)
            for (uint32_t x = 0; x < res; x++) {
                size_t dst = ((size_t)(origin[2] + z) * atlas_dims[1] + origin[1] + y) * atlas_dims[0] + origin[0] + x;
                float v = smp[((size_t)z * res + y) * res + x];
                if (spec.sdf_format == IRT_SDF_F16)
                    atlas16[dst] = f16_bits_round_down(v / scale);
                else
                    atlas32[dst] = v;
            }
}

void Workload::frame_data(uint32_t index, uint32_t debug, irt_frame* f, irt_object* objects, irt_node* nodes,
                          irt_light* out_lights) const {
    M4 vp = view_projection(index);
    M4 prev = index == 0 ? vp : view_projection(index - 1);
    std::memset(f, 0, sizeof(*f));
    f->vp = to_f32(vp);
    f->inv_vp = to_f32(inverse(vp));
    f->previous_vp = to_f32(prev);
    f->previous_inv_vp = to_f32(inverse(prev));
    double eye[3], target[3];
    camera_at(index, eye, target);
    f->camera[0] = (float)eye[0];
    f->camera[1] = (float)eye[1];
    f->camera[2] = (float)eye[2];
    f->camera[3] = 0.f;
    irt_settings s;
    settings(&s);
    const uint32_t generation = 1;  // Scene::load starts at generation 1
    f->size[0] = s.render_width;
    f->size[1] = s.render_height;
    f->size[2] = index;
    f->size[3] = generation;
    f->counts[0] = (uint32_t)lights.size();
    f->counts[1] = s.vpl_count;
    f->counts[2] = s.vpl_max_bounces;
    f->counts[3] = (uint32_t)objs.size();
    f->restir[0] = s.restir_direct_candidates;
    f->restir[1] = s.restir_vpl_candidates;
    f->restir[2] = s.restir_spatial_neighbors;
    f->restir[3] = s.restir_spatial_radius;
    f->temporal[0] = s.temporal_history_weight;
    f->temporal[1] = s.depth_threshold;
    f->temporal[2] = s.normal_threshold;
    f->temporal[3] = (float)s.temporal_max_history;
    f->sdf[0] = (float)s.sdf_max_steps;
    f->sdf[1] = s.sdf_hit_epsilon;
    f->sdf[2] = s.sdf_soft_shadow_k;
    f->sdf[3] = 0.f;
    f->rr[0] = s.vpl_rr_min_survival;
    f->rr[1] = s.vpl_rr_max_survival;
    f->rr[2] = (float)s.restir_max_history;
    f->rr[3] = 0.f;
    // Renderer state starts with previous_generation 0 (src/renderer.rs:1591);
    // frames after the first keep the debug mode and generation.
    f->flags[0] = index > 0 ? 1u : 0u;
    f->flags[1] = index > 0 ? generation : 0u;
    f->flags[2] = debug;
    f->flags[3] = 0u;
    std::vector<float> lo(objs.size() * 3), hi(objs.size() * 3);
    for (uint32_t i = 0; i < objs.size(); i++) {
        const Obj& o = objs[i];
        const MeshDesc& md = mesh_desc[o.mesh];
        irt_mat4 model = to_f32(o.model);
        irt_pack_object(&model, &model, o.mesh, o.material, md.sdf_lo, md.sdf_hi, md.resolution, &objects[i]);
        // World AABB of the transformed SDF bounds corners in f32, like
        // glam's transform_point3 (src/renderer.rs:388-400).
        float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = 0; c < 8; c++) {
            float p[3] = {(c & 1) ? md.sdf_hi[0] : md.sdf_lo[0], (c & 2) ? md.sdf_hi[1] : md.sdf_lo[1],
                          (c & 4) ? md.sdf_hi[2] : md.sdf_lo[2]};
            for (int a = 0; a < 3; a++) {
                float w = model.m[0 * 4 + a] * p[0] + model.m[1 * 4 + a] * p[1] + model.m[2 * 4 + a] * p[2] +
                          model.m[3 * 4 + a];
                l[a] = std::min(l[a], w);
                h[a] = std::max(h[a], w);
            }
        }
        for (int a = 0; a < 3; a++) {
            lo[i * 3 + a] = l[a];
            hi[i * 3 + a] = h[a];
        }
    }
    irt_build_hierarchy(lo.data(), hi.data(), (uint32_t)objs.size(), nodes);
    std::memcpy(out_lights, lights.data(), lights.size() * sizeof(irt_light));
}

void Workload::settings(irt_settings* s) const {
    irt_settings_default(s);
    s->render_width = spec.width;
    s->render_height = spec.height;
    s->vpl_count = spec.vpl_count;
    s->vpl_max_bounces = spec.vpl_bounces;
}

}  // namespace irt

namespace {

uint16_t f32_to_f16_bits_rne(float f) {
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

}  // namespace

namespace irt {

uint16_t f16_bits_rne(float f) { return f32_to_f16_bits_rne(f); }

float f16_bits_to_f32(uint16_t h) {
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

// Largest binary16 value not above v (round toward -inf).
uint16_t f16_bits_round_down(float v) {
    uint16_t h = f32_to_f16_bits_rne(v);
    if (f16_bits_to_f32(h) > v) {
        // Step one ulp toward -inf.
        if (h == 0x0000u) return 0x8001u;
        if (h & 0x8000u) return (uint16_t)(h + 1u);
        return (uint16_t)(h - 1u);
    }
    return h;
}

}  // namespace irt
