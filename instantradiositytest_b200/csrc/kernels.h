// kernels.h — host-side launch descriptors of the lighting and SVGF kernels.
#pragma once
#include <cuda_runtime.h>

#include "../../include/irt.h"
#include "workload.h"

namespace irtd {
// The reference's filtered variant of sample_field (src/renderer.rs:277-286,
// chosen there whenever the adapter can filter R32Float textures): one
// hardware-linear fetch of the atlas at the point (origin + q + .5) / dims in
// normalised coordinates — texel coordinate origin + q + .5 — clamp-to-edge,
// instead of 8 texel loads and f32 weights.  linear == 0 selects the
// point-sampled trilinear of common.wgsl:31-38.
struct FieldFilter {
    cudaTextureObject_t linear;  // the atlas: texel coordinates, linear filter, clamp
    float dims[3];               // atlas extent in texels
};
}  // namespace irtd

// Lighting stages: 0..7 are the reference entry points in schedule order
// (candidates_direct, candidates_indirect, temporal_direct, temporal_indirect,
// spatial_direct, spatial_indirect, resolve_direct, resolve_indirect).
constexpr int kStageReuse = 100;    // fused 0..3
constexpr int kStageShade = 101;    // fused 4..7 with the march inline (one thread per pixel)
constexpr int kStageSpatial = 102;  // fused 4..5 + resolve set-up: emits visibility rays
constexpr int kStageCombine = 103;  // resolve 6..7 from contributions x visibility
constexpr int kStageArchive = 104;  // batched: VPL archive slot copy + ray-counter reset

// A visibility ray of the resolve passes (sdf.wgsl:61-81 arguments), 64 bytes:
//   a = (p.xyz, bits(pixel * 2 + kind))  kind 0 = direct, 1 = indirect
//   b = (n.xyz, 1 if the endpoint is offset along end_normal else 0)
//   c = (target.xyz, 0), d = (end_normal.xyz, 0)
struct RayRecord {
    float4 a, b, c, d;
};

struct LightingLaunch {
    const irt_frame* frame;
    irt_gbuffer gbuffer;
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    const irt_light* lights;
    cudaTextureObject_t atlas;
    int sdf_f16;
    const void* sdf_cells;  // corner cells of the field meshes (dev_sdf.cuh), or null
    irtd::FieldFilter field_filter;
    uint32_t* error;
    const irt_vpl* cur_vpls;
    const irt_vpl* prev_vpls;
    const irt_vpl* archive;
    const float* prev_depth;
    const void* prev_normal;
    irt_reservoir* dres[3];
    irt_reservoir* ires[3];
    float4* direct_out;
    void* noisy_out;
    int radiance_f16;
    int keep_candidates;
    const float4* guide;      // world positions of this frame's pixels
    const float4* old_guide;  // ... of the previous frame's pixels
    const float4* feat;       // decoded normal/colour/params of this frame's pixels (f16, packed), or null
    // ray-queue resolve (kStageSpatial / march / kStageCombine)
    RayRecord* rays;         // capacity 2 * W * H
    uint32_t* ray_counters;  // [0] VPL rays (queue front), [1] rays fetched by the march, [2] light rays (back)
    float* vis;              // visibility per pixel * 2 + kind
    float4* pending;         // per pixel: direct contribution (w = 1: x vis), indirect (w = 1: x vis)
};

struct MarchLaunch {
    const irt_frame* frame;
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    cudaTextureObject_t atlas;
    int sdf_f16;
    const void* sdf_cells;  // corner cells of the field meshes (dev_sdf.cuh), or null
    irtd::FieldFilter field_filter;
    uint32_t* error;
    const float4* march_scene;  // compact nodes + objects (irt_march_scene_bytes)
    // Leaf-order cache: a kGridRes^3 grid over the root box; per cell the
    // first kCellEntries objects by increasing distance from the cell to their
    // BVH leaf box, with those distances and the next one as a sentinel.
    const uint4* cells;
    float grid_org[3], grid_inv[3];
    const RayRecord* rays;
    uint32_t* ray_counters;
    float* vis;
    int num_sms;
    int fast;  // 1: approximate division / square root build (march_fast.cu)
};
cudaError_t irt_launch_march(const MarchLaunch& M, cudaStream_t st);
// Bytes of the compact march scene of `object_count` objects: 2N-1 nodes of
// 32 bytes, then N object records of 176 bytes (mesh folded in).
uint32_t irt_march_scene_bytes(uint32_t object_count);
constexpr uint32_t kMaxMarchObjects = 1024;  // the march scene lives in shared memory
constexpr uint32_t kGridRes = 32;
constexpr uint32_t kCellEntries = 8;
// One cell: 4 x uint4 = ids (8 x u16 in words 0-3), lower bounds (f32 words
// 4-11), sentinel bound of the first object left out (word 12), pad.
constexpr uint32_t kCellWords = 16;
// Leaf-order cache build (leafcache.cu) from the staged march scene.
struct LeafCacheLaunch {
    const float4* march_scene;  // nodes + object records on the device
    uint32_t n;                 // objects
    cudaTextureObject_t atlas;
    int sdf_f16;
    const void* sdf_cells;  // corner cells of the field meshes (dev_sdf.cuh), or null
    irtd::FieldFilter field_filter;
    double grid_org_d[3], grid_size_d[3];
    float* corners;             // (kGridRes+1)^3 * n floats, or null: box bounds only
    uint32_t* cells;            // kGridRes^3 * kCellWords words
};
cudaError_t irt_launch_leaf_cache(const LeafCacheLaunch& L, cudaStream_t st);
constexpr uint32_t kMaxCornerObjects = 256;  // corner bounds for scenes up to this many objects

struct SvgfLaunch {
    const irt_frame* frame;
    irt_gbuffer gbuffer;
    const float* old_depth;
    const void* old_normal;
    const void* in;          // temporal: noisy; variance/atrous: input radiance
    const void* aux;         // temporal: old radiance (feedback)
    const void* moments_in;  // temporal: old moments; variance: current moments
    void* out;
    void* out2;              // atrous: optional second output
    void* moments_out;       // temporal: current moments
    int step;
    int radiance_f16;
    int moments_f16;          // moments: 0 float4 (E[l], E[l^2], age, 0); 1 MomF16 (half mean, half deviation, f32 age)
    const float4* guide;      // per-pixel positions of this frame (or null)
    const float4* old_guide;  // ... of the previous frame (or null)
    const float4* feat;       // per-pixel edge-stopping features (or null)
};
// irt_launch_svgf stages: 0 temporal, 1 variance, 2 a-trous, 3 position guide
// of this frame (out = float4[W*H]), 4 guide of the previous frame (from
// old_depth and previous_inv_vp), 6 guide of this frame (out) and its
// edge-stopping features (out2 = float4[2*W*H]).

// VPL paths of one frame (vplgen.cu): lights on the device, ray casts
// against a workload's primitive table.
struct VplLaunch {
    const irt_frame* frame;
    irt::PrimTable prims;
    const irt_light* lights;
    irt_vpl* out;
};
cudaError_t irt_launch_vpls(const VplLaunch& L, cudaStream_t st);
// The workload's flattened primitive table and triangle tables on the
// current device (built on first use and kept with the workload).
cudaError_t irt_workload_prims(const irt_workload* wl, irt::PrimTable* out);

cudaError_t irt_launch_lighting(const LightingLaunch& L, int stage, cudaStream_t st);

// Corner cells of one field mesh (sdfcells.cu): records [base, base +
// (res-1)^3) of `out` from the atlas tile at `origin` (DevScene::sdf_cells).
cudaError_t irt_pack_sdf_cells(cudaTextureObject_t atlas, int f16, const uint32_t origin[3], uint32_t res,
                               uint64_t base, void* out, cudaStream_t st);
// sample_field of the mesh `row` (its device row values: hi[3] = first
// corner cell) at n grid-space points q (3 floats each); out: n floats.
namespace irtd {
struct DevScene;
}
cudaError_t irt_launch_sample_field(const irtd::DevScene& sc, const irt_mesh& row, const float* q, uint32_t n,
                                    float* out, cudaStream_t st);

// ------------------------------------------------------------------ batched views
// One launch per pass over the views of a batch.  `table` is a device array
// of n per-view argument records of the stage (lighting: the LightArgs of
// irt_lighting_args_fill; SVGF: the records of irt_svgf_view_fill),
// `frames` the n per-view frames on the device, `tile_start` n+1 block
// offsets (2-D kernels: tiles of bx x by pixels; 1-D kernels: 256 pixels).
struct BatchLaunch {
    uint32_t n;
    const irt_frame* frames;
    const void* table;
    const uint32_t* tile_start;
    uint32_t tiles;
    uint32_t bx, by;
    int gbuffer_format;
    int radiance_f16, moments_f16;
    int keep;
};
size_t irt_lighting_args_size(int gbuffer_format);
void irt_lighting_args_fill(const LightingLaunch& L, void* out);
cudaError_t irt_launch_lighting_batched(const BatchLaunch& B, int stage, cudaStream_t st);
// SVGF stages of a batch: 0 temporal, 1 variance, 2 a-trous (records carry
// the step), 3 guides of this frame, 4 guides of the previous frame, 5 depth
// and normal history copy, 6 guides and features of this frame.
size_t irt_svgf_view_size(int gbuffer_format);
void irt_svgf_view_fill(const SvgfLaunch& L, void* out);
cudaError_t irt_launch_svgf_batched(const BatchLaunch& B, int stage, cudaStream_t st);
cudaError_t irt_launch_svgf_spatial_batched(const BatchLaunch& B, int stage, cudaStream_t st);

// Batched march: views grouped by scene; each group's compact scene is
// staged in shared memory once per CTA and the group's ray queues (one per
// view) are consumed in order.
struct MarchQueue {
    const RayRecord* rays;
    uint32_t* counters;  // [0] rays at the front, [1] rays fetched, [2] rays at the back
    float* vis;
    uint32_t cap;        // records (2 * W * H)
};
struct alignas(16) MarchGroup {
    irt_frame f;                // counts[3] and sdf[] of the group's views
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    cudaTextureObject_t atlas;
    int sdf_f16;
    const void* sdf_cells;  // corner cells of the field meshes (dev_sdf.cuh), or null
    irtd::FieldFilter field_filter;
    uint32_t* error;
    const float4* march_scene;
    uint32_t scene_vec4;
    const uint4* cells;
    float grid_org[3], grid_inv[3];
    uint32_t q_begin, q_end;    // the group's queues in the queue table
};
struct MarchBatch {
    uint32_t n_groups;
    const MarchGroup* groups;   // device
    const MarchQueue* queues;   // device
    uint32_t max_scene_bytes;
    int num_sms;
    int blocks_per_sm;          // 0 = occupancy maximum
    int fast;
};
cudaError_t irt_launch_march_batched(const MarchBatch& M, cudaStream_t st);
// Lights with the spot direction normalised and cos(angle / 2) in
// direction_angle, the form the lighting kernels read.
cudaError_t irt_launch_prepare_lights(const irt_light* lights, uint32_t n, irt_light* out, cudaStream_t st);
cudaError_t irt_launch_svgf(const SvgfLaunch& L, int stage, cudaStream_t st);
// Stages 1 (variance) and 2 (a-trous), the fast-math SVGF passes.
cudaError_t irt_launch_svgf_spatial(const SvgfLaunch& L, int stage, cudaStream_t st);
