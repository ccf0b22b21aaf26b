// tri_bvh.cpp — host builder and CPU caster of the per-mesh triangle
// hierarchies (layout in tri_bvh.h).
#include "tri_bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace irt {

void build_tri_bvh(const irt_vertex* vertices, const uint32_t* indices, uint32_t index_count, TriBvh& out) {
    const uint32_t n = index_count / 3;
    out.nodes.clear();
    out.tris.clear();
    if (n == 0) return;
    std::vector<float> cen((size_t)n * 3), blo((size_t)n * 3), bhi((size_t)n * 3);
    for (uint32_t i = 0; i < n; i++) {
        for (int a = 0; a < 3; a++) {
            float p0 = vertices[indices[i * 3]].position[a], p1 = vertices[indices[i * 3 + 1]].position[a],
                  p2 = vertices[indices[i * 3 + 2]].position[a];
            blo[i * 3 + a] = std::min(p0, std::min(p1, p2));
            bhi[i * 3 + a] = std::max(p0, std::max(p1, p2));
            cen[i * 3 + a] = (blo[i * 3 + a] + bhi[i * 3 + a]) * .5f;
        }
    }
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    struct Task {
        uint32_t node, begin, end;
    };
    out.nodes.reserve(2 * (n / kTriLeaf + 1));
    out.nodes.push_back(TriNode{});
    std::vector<Task> tasks{{0, 0, n}};
    while (!tasks.empty()) {
        Task k = tasks.back();
        tasks.pop_back();
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t j = k.begin; j < k.end; j++) {
            uint32_t t = order[j];
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], blo[t * 3 + a]);
                hi[a] = std::max(hi[a], bhi[t * 3 + a]);
                clo[a] = std::min(clo[a], cen[t * 3 + a]);
                chi[a] = std::max(chi[a], cen[t * 3 + a]);
            }
        }
        TriNode& nd = out.nodes[k.node];
        for (int a = 0; a < 3; a++) {
            nd.lo[a] = lo[a];
            nd.hi[a] = hi[a];
        }
        const uint32_t count = k.end - k.begin;
        if (count <= kTriLeaf) {
            nd.first = k.begin;
            nd.count = count;
            continue;
        }
        int axis = 0;
        for (int a = 1; a < 3; a++)
            if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
        const uint32_t mid = k.begin + count / 2;
        std::nth_element(order.begin() + k.begin, order.begin() + mid, order.begin() + k.end,
                         [&](uint32_t x, uint32_t y) {
                             float cx = cen[x * 3 + axis], cy = cen[y * 3 + axis];
                             return cx < cy || (cx == cy && x < y);
                         });
        const uint32_t left = (uint32_t)out.nodes.size();
        out.nodes.push_back(TriNode{});
        out.nodes.push_back(TriNode{});
        out.nodes[k.node].first = left;
        out.nodes[k.node].count = 0;
        tasks.push_back(Task{left + 1, mid, k.end});
        tasks.push_back(Task{left, k.begin, mid});
    }
    // Triangle records in leaf order.
    out.tris.resize(n);
    for (uint32_t j = 0; j < n; j++) {
        const uint32_t t = order[j];
        const irt_vertex* v[3] = {&vertices[indices[t * 3]], &vertices[indices[t * 3 + 1]],
                                  &vertices[indices[t * 3 + 2]]};
        TriRec& r = out.tris[j];
        float e1[3], e2[3];
        for (int a = 0; a < 3; a++) {
            r.v0[a] = v[0]->position[a];
            e1[a] = v[1]->position[a] - v[0]->position[a];
            e2[a] = v[2]->position[a] - v[0]->position[a];
            r.e1[a] = e1[a];
            r.e2[a] = e2[a];
        }
        const float g[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        float nn[3][3];
        for (int c = 0; c < 3; c++) {
            const float* src = v[c]->normal;
            float l = std::sqrt(src[0] * src[0] + src[1] * src[1] + src[2] * src[2]);
            const float* use = src;
            if (!(l > 0.f)) {
                use = g;
                l = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
                if (!(l > 0.f)) l = 1.f;
            }
            for (int a = 0; a < 3; a++) nn[c][a] = use[a] / l;
        }
        r.v0[3] = nn[0][0];
        r.e1[3] = nn[0][1];
        r.e2[3] = nn[0][2];
        for (int a = 0; a < 3; a++) {
            r.n1[a] = nn[1][a];
            r.n2[a] = nn[2][a];
        }
        r.n1[3] = r.n2[3] = 0.f;
    }
}

namespace {
bool ray_box(const float lo[3], const float hi[3], const double o[3], const double inv[3], double tmin, double tmax) {
    for (int a = 0; a < 3; a++) {
        double t0 = (lo[a] - o[a]) * inv[a], t1 = (hi[a] - o[a]) * inv[a];
        if (t0 > t1) std::swap(t0, t1);
        tmin = std::max(tmin, t0);
        tmax = std::min(tmax, t1);
        if (!(tmin <= tmax)) return false;
    }
    return true;
}
}  // namespace

bool cast_tri_bvh(const TriBvh& b, const double o[3], const double d[3], double tmin, double tmax, bool cull,
                  double& t_out, double n_out[3]) {
    if (b.nodes.empty()) return false;
    double inv[3];
    for (int a = 0; a < 3; a++) inv[a] = 1.0 / d[a];
    uint32_t stack[kTriStack];
    uint32_t sp = 0;
    stack[sp++] = 0;
    int hit = -1;
    double bu = 0, bv = 0;
    while (sp) {
        const TriNode& nd = b.nodes[stack[--sp]];
        if (!ray_box(nd.lo, nd.hi, o, inv, tmin, tmax)) continue;
        if (nd.count == 0) {
            if (sp + 2 > kTriStack) continue;  // unreachable for hierarchies built above
            stack[sp++] = nd.first + 1;
            stack[sp++] = nd.first;
            continue;
        }
        for (uint32_t j = nd.first; j < nd.first + nd.count; j++) {
            const TriRec& r = b.tris[j];
            const double e1[3] = {r.e1[0], r.e1[1], r.e1[2]}, e2[3] = {r.e2[0], r.e2[1], r.e2[2]};
            if (cull) {
                const double g[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                     e1[0] * e2[1] - e1[1] * e2[0]};
                if (g[0] * d[0] + g[1] * d[1] + g[2] * d[2] >= 0.0) continue;
            }
            const double p[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
            const double det = e1[0] * p[0] + e1[1] * p[1] + e1[2] * p[2];
            if (det == 0.0) continue;
            const double id = 1.0 / det;
            const double s[3] = {o[0] - r.v0[0], o[1] - r.v0[1], o[2] - r.v0[2]};
            const double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * id;
            if (u < 0.0 || u > 1.0) continue;
            const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
            const double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * id;
            if (v < 0.0 || u + v > 1.0) continue;
            const double t = (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) * id;
            if (t > tmin && t < tmax) {
                tmax = t;
                hit = (int)j;
                bu = u;
                bv = v;
            }
        }
    }
    if (hit < 0) return false;
    const TriRec& r = b.tris[(size_t)hit];
    const double w0 = 1.0 - bu - bv;
    const double n0[3] = {r.v0[3], r.e1[3], r.e2[3]};
    for (int a = 0; a < 3; a++) n_out[a] = n0[a] * w0 + r.n1[a] * bu + r.n2[a] * bv;
    t_out = tmax;
    return true;
}

}  // namespace irt
