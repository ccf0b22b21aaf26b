// host_scene.cpp — host logic of the reference renderer that builds the data
// the lighting path consumes: settings validation, mesh metadata, SDF atlas
// tiling, per-object records and the stackless BVH.  Compiled with
// -ffp-contract=off so f32 arithmetic follows the reference's Rust (which
// never contracts).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "host_math.h"

using namespace irt;

namespace {

struct F3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline F3 f3(const float* p) { return F3{p[0], p[1], p[2]}; }
inline float len_sq(F3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline float len(F3 a) { return std::sqrt(len_sq(a)); }

// f32::total_cmp ordering key.
inline int32_t total_key(float f) {
    int32_t i;
    std::memcpy(&i, &f, 4);
    return i ^ (int32_t)((uint32_t)(i >> 31) >> 1);
}

struct Bound {
    uint32_t id;
    F3 lo, hi;
};

// build() of hierarchy() (src/renderer.rs:404-450): preorder node, children
// split at the median of the centroid order along the longest axis, escape
// index = node count after the subtree.
uint32_t build_node(Bound* b, size_t n, std::vector<irt_node>& nodes) {
    uint32_t index = (uint32_t)nodes.size();
    nodes.push_back(irt_node{});
    F3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = 0; i < n; i++) {
        lo = F3{std::min(lo.x, b[i].lo.x), std::min(lo.y, b[i].lo.y), std::min(lo.z, b[i].lo.z)};
        hi = F3{std::max(hi.x, b[i].hi.x), std::max(hi.y, b[i].hi.y), std::max(hi.z, b[i].hi.z)};
    }
    uint32_t meta[4];
    if (n == 1) {
        meta[0] = b[0].id;
        meta[1] = 0;
        meta[2] = 1;
        meta[3] = 0;
    } else {
        F3 e{hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
        int axis = (e.x > e.y && e.x > e.z) ? 0 : (e.y > e.z ? 1 : 2);
        std::stable_sort(b, b + n, [axis](const Bound& a, const Bound& c) {
            float ka = a.lo[axis] + a.hi[axis];
            float kc = c.lo[axis] + c.hi[axis];
            return total_key(ka) < total_key(kc);
        });
        size_t half = n / 2;
        uint32_t left = build_node(b, half, nodes);
        uint32_t right = build_node(b + half, n - half, nodes);
        meta[0] = left;
        meta[1] = right;
        meta[2] = 0;
        meta[3] = 0;
    }
    meta[3] = (uint32_t)nodes.size();
    irt_node& node = nodes[index];
    node.lo[0] = lo.x;
    node.lo[1] = lo.y;
    node.lo[2] = lo.z;
    node.lo[3] = 0.f;
    node.hi[0] = hi.x;
    node.hi[1] = hi.y;
    node.hi[2] = hi.z;
    node.hi[3] = 0.f;
    std::memcpy(node.info, meta, sizeof(meta));
    return index;
}

}  // namespace

extern "C" {

void irt_settings_default(irt_settings* s) {
    std::memset(s, 0, sizeof(*s));
    s->render_width = 1920;
    s->render_height = 1200;
    s->vpl_count = 100;
    s->vpl_max_bounces = 3;
    s->vpl_rr_min_survival = 0.1f;
    s->vpl_rr_max_survival = 0.95f;
    s->restir_direct_candidates = 8;
    s->restir_vpl_candidates = 8;
    s->restir_spatial_neighbors = 4;
    s->restir_spatial_radius = 12;
    s->restir_max_history = 4;
    s->svgf_iterations = 4;
    s->depth_threshold = 0.03f;
    s->normal_threshold = 0.85f;
    s->temporal_history_weight = 0.9f;
    s->temporal_max_history = 32;
    s->sdf_max_steps = 96;
    s->sdf_hit_epsilon = 0.001f;
    s->sdf_soft_shadow_k = 16.0f;
    s->target_frame_ms = 8.0f;
}

// Settings::validate (src/settings.rs:42-105): same rules, same messages.
irt_status irt_settings_validate(const irt_settings* s, char* msg, size_t msg_len) {
    auto fail = [&](const char* m) {
        if (msg && msg_len) std::snprintf(msg, msg_len, "%s", m);
        return IRT_E_INVALID;
    };
    if (!s) return fail("null settings");
    if (!(s->render_width > 0 && s->render_height > 0 && s->render_width <= 8192 && s->render_height <= 8192))
        return fail("invalid render size");
    if (!(s->vpl_count > 0 && s->vpl_count <= 65536 && s->vpl_max_bounces >= 1 && s->vpl_max_bounces <= 32))
        return fail("invalid VPL budget");
    if (!(s->vpl_rr_min_survival > 0.f && s->vpl_rr_max_survival < 1.f &&
          s->vpl_rr_min_survival <= s->vpl_rr_max_survival))
        return fail("invalid roulette probabilities");
    if (!(s->restir_direct_candidates > 0 && s->restir_vpl_candidates > 0 && s->restir_direct_candidates <= 256 &&
          s->restir_vpl_candidates <= 256 && s->restir_spatial_neighbors <= 32 && s->restir_spatial_radius <= 256))
        return fail("invalid ReSTIR settings");
    if (!(s->restir_max_history > 0 && s->restir_max_history <= 32 && s->svgf_iterations > 0 &&
          s->svgf_iterations <= 5))
        return fail("invalid ReSTIR history/SVGF iteration count");
    if (!(s->temporal_history_weight >= 0.f && s->temporal_history_weight < 1.f && s->temporal_max_history > 0 &&
          s->temporal_max_history <= 256))
        return fail("invalid temporal settings");
    if (!(s->sdf_max_steps > 0 && s->sdf_max_steps <= 1024 && s->sdf_hit_epsilon > 0.f &&
          std::isfinite(s->sdf_hit_epsilon) && s->sdf_soft_shadow_k > 0.f && std::isfinite(s->sdf_soft_shadow_k)))
        return fail("invalid SDF settings");
    if (!(s->depth_threshold > 0.f && std::isfinite(s->depth_threshold) && s->normal_threshold >= 0.f &&
          s->normal_threshold <= 1.f && s->target_frame_ms > 0.f && std::isfinite(s->target_frame_ms)))
        return fail("invalid rejection/frame budget");
    if (msg && msg_len) msg[0] = 0;
    return IRT_OK;
}

// is_box_geometry (src/renderer.rs:287-329): a 12-triangle mesh whose
// vertices sit on the AABB corners and whose faces each tile one box side
// with two triangles sharing a face diagonal.
int32_t irt_is_box_geometry(const irt_vertex* vertices, uint32_t vertex_count, const uint32_t* indices,
                            uint32_t index_count, const float lo_[3], const float hi_[3]) {
    F3 lo = f3(lo_), hi = f3(hi_);
    if (index_count != 36) return 0;
    float ext_min = std::min(hi.x - lo.x, std::min(hi.y - lo.y, hi.z - lo.z));
    if (ext_min <= 0.f) return 0;
    std::vector<uint8_t> corners(vertex_count);
    for (uint32_t v = 0; v < vertex_count; v++) {
        F3 p = f3(vertices[v].position);
        uint8_t corner = 0;
        for (int axis = 0; axis < 3; axis++) {
            if (p[axis] == hi[axis])
                corner |= (uint8_t)(1u << axis);
            else if (p[axis] != lo[axis])
                return 0;
        }
        corners[v] = corner;
    }
    std::vector<std::array<uint8_t, 3>> faces[6];
    for (uint32_t t = 0; t < 12; t++) {
        std::array<uint8_t, 3> c;
        for (int k = 0; k < 3; k++) {
            uint32_t i = indices[t * 3 + k];
            if (i >= vertex_count) return 0;
            c[k] = corners[i];
        }
        std::sort(c.begin(), c.end());
        if (c[0] == c[1] || c[1] == c[2]) return 0;
        int axis = -1;
        for (int a = 0; a < 3 && axis < 0; a++) {
            uint8_t mask = (uint8_t)(1u << a);
            if ((c[0] & mask) == (c[1] & mask) && (c[0] & mask) == (c[2] & mask)) axis = a;
        }
        if (axis < 0) return 0;
        int side = (c[0] >> axis) & 1;
        faces[axis * 2 + side].push_back(c);
    }
    for (int f = 0; f < 6; f++) {
        if (faces[f].size() != 2) return 0;
        uint8_t shared[3];
        int ns = 0;
        for (uint8_t c : faces[f][0])
            if (std::find(faces[f][1].begin(), faces[f][1].end(), c) != faces[f][1].end()) shared[ns++] = c;
        if (ns != 2) return 0;
        if (__builtin_popcount((unsigned)(shared[0] ^ shared[1])) != 2) return 0;
    }
    return 1;
}

// field_lipschitz_bound (src/renderer.rs:330-358): the largest corner
// finite-difference gradient over every cell that can yield a positive
// marching distance, at least 1, times 1.0001.
float irt_field_lipschitz_bound(const float* samples, uint32_t resolution, const float spacing_[3]) {
    size_t n = resolution;
    F3 spacing = f3(spacing_);
    float positive_threshold = len(spacing) * (0.5f + 1.f / 128.f);
    float maximum_squared = 1.f;
    for (size_t z = 0; z + 1 < n; z++)
        for (size_t y = 0; y + 1 < n; y++)
            for (size_t x = 0; x + 1 < n; x++) {
                float values[8];
                bool all_below = true;
                for (size_t i = 0; i < 8; i++) {
                    values[i] = samples[(x + (i & 1)) + n * ((y + ((i >> 1) & 1)) + n * (z + (i >> 2)))];
                    if (!(values[i] <= positive_threshold)) all_below = false;
                }
                if (all_below) continue;
                for (size_t corner = 0; corner < 8; corner++) {
                    float dx = (values[(corner & 6) | 1] - values[corner & 6]) / spacing.x;
                    float dy = (values[(corner & 5) | 2] - values[corner & 5]) / spacing.y;
                    float dz = (values[(corner & 3) | 4] - values[corner & 3]) / spacing.z;
                    float sq = dx * dx + dy * dy + dz * dz;
                    maximum_squared = std::max(maximum_squared, sq);
                }
            }
    return std::sqrt(maximum_squared) * 1.0001f;
}

// Renderer::new per-mesh metadata (src/renderer.rs:835-885).
irt_status irt_mesh_metadata(const irt_vertex* vertices, uint32_t vertex_count, const uint32_t* indices,
                             uint32_t index_count, const float* samples, uint32_t resolution,
                             const float bounds_min[3], const float bounds_max[3],
                             const uint32_t atlas_origin[3], irt_mesh* out) {
    if (!vertices || !vertex_count || !samples || resolution < 2 || !out) return IRT_E_INVALID;
    std::memset(out, 0, sizeof(*out));
    float res1 = (float)(resolution - 1);
    F3 spacing{(bounds_max[0] - bounds_min[0]) / res1, (bounds_max[1] - bounds_min[1]) / res1,
               (bounds_max[2] - bounds_min[2]) / res1};
    F3 glo{INFINITY, INFINITY, INFINITY}, ghi{-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t v = 0; v < vertex_count; v++) {
        F3 p = f3(vertices[v].position);
        glo = F3{std::min(glo.x, p.x), std::min(glo.y, p.y), std::min(glo.z, p.z)};
        ghi = F3{std::max(ghi.x, p.x), std::max(ghi.y, p.y), std::max(ghi.z, p.z)};
    }
    F3 center{(glo.x + ghi.x) * 0.5f, (glo.y + ghi.y) * 0.5f, (glo.z + ghi.z) * 0.5f};
    float radius = 0.f;
    for (uint32_t v = 0; v < vertex_count; v++) {
        F3 p = f3(vertices[v].position);
        F3 d{p.x - center.x, p.y - center.y, p.z - center.z};
        radius = std::max(radius, len(d));
    }
    radius = radius * 1.000001f + 0.000001f;
    for (int i = 0; i < 3; i++) {
        out->lo[i] = bounds_min[i];
        out->hi[i] = bounds_max[i];
    }
    out->geometry[0] = 0;
    out->geometry[1] = vertex_count;
    out->geometry[2] = 0;
    out->geometry[3] = index_count;
    out->field[0] = atlas_origin[0];
    out->field[1] = atlas_origin[1];
    out->field[2] = atlas_origin[2];
    out->field[3] = resolution;
    out->grid[0] = 1.f / spacing.x;
    out->grid[1] = 1.f / spacing.y;
    out->grid[2] = 1.f / spacing.z;
    out->grid[3] = len(spacing);
    out->geometry_lo[0] = glo.x;
    out->geometry_lo[1] = glo.y;
    out->geometry_lo[2] = glo.z;
    out->geometry_lo[3] = irt_is_box_geometry(vertices, vertex_count, indices, index_count, &glo.x, &ghi.x) ? 1.f : 0.f;
    out->geometry_hi[0] = ghi.x;
    out->geometry_hi[1] = ghi.y;
    out->geometry_hi[2] = ghi.z;
    float spacing_arr[3] = {spacing.x, spacing.y, spacing.z};
    out->geometry_hi[3] = 1.f / irt_field_lipschitz_bound(samples, resolution, spacing_arr);
    out->enclosing_sphere[0] = center.x;
    out->enclosing_sphere[1] = center.y;
    out->enclosing_sphere[2] = center.z;
    out->enclosing_sphere[3] = radius;
    return IRT_OK;
}

// Atlas tiling (src/renderer.rs:778-795).
void irt_atlas_layout(uint32_t count, uint32_t tile, uint32_t grid_out[3], uint32_t extent_out[3]) {
    uint32_t gx = 1;
    while (gx * gx * gx < count) gx++;
    uint32_t gy = 1;
    while (gx * gy * gy < count) gy++;
    uint32_t gz = (count + gx * gy - 1) / (gx * gy);
    if (gz == 0) gz = 1;
    grid_out[0] = gx;
    grid_out[1] = gy;
    grid_out[2] = gz;
    extent_out[0] = tile * gx;
    extent_out[1] = tile * gy;
    extent_out[2] = tile * gz;
}

// hierarchy() (src/renderer.rs:385-455).
irt_status irt_build_hierarchy(const float* object_lo, const float* object_hi, uint32_t count, irt_node* nodes_out) {
    if (count == 0 || !object_lo || !object_hi || !nodes_out) return IRT_E_INVALID;
    std::vector<Bound> b(count);
    for (uint32_t i = 0; i < count; i++) b[i] = Bound{i, f3(object_lo + 3 * i), f3(object_hi + 3 * i)};
    std::vector<irt_node> nodes;
    nodes.reserve(2 * (size_t)count);
    build_node(b.data(), b.size(), nodes);
    std::memcpy(nodes_out, nodes.data(), nodes.size() * sizeof(irt_node));
    return IRT_OK;
}

// objects() (src/renderer.rs:359-384): model, previous, inverse and
// [mesh, material, bits(scale), bits(|spacing| * scale)] where scale is the
// length of the model's first column.
void irt_pack_object(const irt_mat4* model, const irt_mat4* previous, uint32_t mesh_id, uint32_t material_id,
                     const float sdf_lo[3], const float sdf_hi[3], uint32_t sdf_resolution, irt_object* out) {
    out->model = *model;
    out->previous = *previous;
    out->inverse = to_f32(inverse(from_f32(*model)));
    float res1 = (float)(sdf_resolution - 1);
    F3 spacing{(sdf_hi[0] - sdf_lo[0]) / res1, (sdf_hi[1] - sdf_lo[1]) / res1, (sdf_hi[2] - sdf_lo[2]) / res1};
    F3 x_axis{model->m[0], model->m[1], model->m[2]};
    float scale = len(x_axis);
    out->info[0] = mesh_id;
    out->info[1] = material_id;
    out->info[2] = f32_bits(scale);
    out->info[3] = f32_bits(len(spacing) * scale);
}

}  // extern "C"

