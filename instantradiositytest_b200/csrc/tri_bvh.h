// tri_bvh.h — per-mesh triangle hierarchies for the input producers of
// loaded scenes: the G-buffer producer (stands in for the gbuffer.wgsl
// raster, src/renderer.rs:1801-1862) and the VPL generator (stands in for the
// ray query of vpl.wgsl:17-22 against the scene's acceleration structure).
//
// Layout shared by the host builder, the CPU caster and the CUDA caster:
//   TriNode  32 B: a = (lo.xyz, bits(first)), b = (hi.xyz, bits(count));
//            count == 0: inner node, children at `first` and `first + 1`;
//            count > 0: leaf over tris [first, first + count).
//   TriRec   80 B: v0 (w = n0.x), e1 = v1 - v0 (w = n0.y), e2 = v2 - v0
//            (w = n0.z), n1, n2 — unit vertex normals in mesh space.
// Inner nodes are split at the median centroid of their longest axis, so a
// hierarchy over n triangles is at most ceil(log2(n)) + 1 levels deep.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/irt.h"

namespace irt {

constexpr uint32_t kTriLeaf = 4;     // triangles per leaf at most
constexpr uint32_t kTriStack = 64;   // traversal stack entries (depth bound above)

struct TriNode {
    float lo[3];
    uint32_t first;
    float hi[3];
    uint32_t count;
};
struct TriRec {
    float v0[4], e1[4], e2[4], n1[4], n2[4];
};
static_assert(sizeof(TriNode) == 32, "TriNode layout");
static_assert(sizeof(TriRec) == 80, "TriRec layout");

struct TriBvh {
    std::vector<TriNode> nodes;
    std::vector<TriRec> tris;
};

// Builds the hierarchy of a non-empty triangle list (indices into vertices,
// already validated).  Vertex normals are normalised; a zero normal becomes
// the triangle's geometric normal.
void build_tri_bvh(const irt_vertex* vertices, const uint32_t* indices, uint32_t index_count, TriBvh& out);

// Nearest hit t in (tmin, tmax) along o + t d in mesh space (Moller-Trumbore
// in double).  `cull` skips triangles whose geometric normal faces along d
// (back faces of counter-clockwise fronts, as the raster's Face::Back cull).
// On a hit: t, the barycentric-interpolated vertex normal (not normalised).
bool cast_tri_bvh(const TriBvh& b, const double o[3], const double d[3], double tmin, double tmax, bool cull,
                  double& t, double n[3]);

}  // namespace irt
