// workload.h — seeded procedural room workloads (host side).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/irt.h"
#include "host_math.h"
#include "tri_bvh.h"

namespace irt {

struct Part {  // one analytic solid of a mesh, in mesh-local space
    bool sphere = false;
    double radius = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
};

struct MeshDesc {
    std::vector<Part> parts;
    std::vector<irt_vertex> vertices;
    std::vector<uint32_t> indices;
    float sdf_lo[3], sdf_hi[3];
    uint32_t resolution = 0;  // SDF samples per axis
    // Meshes of a loaded scene file are triangle lists: ray casts run
    // against their hierarchy instead of analytic parts.
    bool triangles = false;
    TriBvh bvh;
};

struct Obj {
    uint32_t mesh, material;
    M4 model, inv_model;
};

struct Workload {
    irt_workload_spec spec{};
    std::vector<MeshDesc> mesh_desc;
    std::vector<Obj> objs;
    std::vector<irt_material> materials;
    std::vector<irt_light> lights;
    std::vector<irt_mesh> meshes;
    std::vector<float> atlas32;
    std::vector<uint16_t> atlas16;
    uint32_t atlas_dims[3] = {0, 0, 0}, atlas_grid[3] = {0, 0, 0};
    uint32_t path_frames = 64;
    double angle0 = 0;
    // A scene loaded from a manifest keeps its camera fixed (Camera::matrix,
    // src/scene.rs:119-128); procedural rooms follow the orbit path.
    bool loaded = false;
    double cam_eye[3] = {0, 0, 0};
    double cam_q[4] = {0, 0, 0, 1};
    double cam_fov = 0, cam_near = 0, cam_far = 0;
    // Device copy of the primitive table and the triangle hierarchies for
    // the CUDA input producers (lazily created, owned here).
    void* dev_prims = nullptr;
    void* dev_nodes = nullptr;
    void* dev_tris = nullptr;
    int dev_prims_device = -1;
    // Frees the device tables above; set by the CUDA producers when they
    // upload them (the host-only library never does).
    void (*release_device)(Workload&) = nullptr;
    uint32_t dev_prims_count = 0;

    bool build();
    // Writes mesh m's SDF samples (res^3, x fastest) into its atlas tile at
    // `origin`: f32 texels as they are, or f16 texels of value / scale
    // rounded toward -inf with scale = the voxel diagonal (kept in
    // meshes[m].lo[3]) so the dequantised field never exceeds the f32 one.
    void store_field(uint32_t m, const float* samples, uint32_t res, const uint32_t origin[3]);
    void camera_at(uint32_t frame, double eye[3], double target[3]) const;
    M4 view_projection(uint32_t frame) const;
    void frame_data(uint32_t index, uint32_t debug, irt_frame* f, irt_object* objects, irt_node* nodes,
                    irt_light* lights) const;
    void settings(irt_settings* s) const;
    // `cull` skips back-facing triangles (primary rays of the raster);
    // analytic parts only report front entries either way.
    bool intersect_object(uint32_t oi, const double o[3], const double d[3], double tmin, double tmax, double& t,
                          double n[3], bool cull = false) const;
    bool cast(const double o[3], const double d[3], double tmin, double tmax, double& t, double n[3],
              uint32_t& object, bool cull = false) const;
};

uint16_t f16_bits_rne(float f);
float f16_bits_to_f32(uint16_t h);
uint16_t f16_bits_round_down(float v);

// Octahedral unit-vector encoding to two snorm16 (Cigolle et al. 2014).
uint32_t oct_encode_snorm16(float x, float y, float z);
// rgba8 unorm packing with round-to-nearest.
uint32_t pack_unorm8x4(float r, float g, float b, float a);

// Flattened primitive record used by the CUDA input producers.
enum : uint32_t { kPrimBox = 0, kPrimSphere = 1, kPrimTriangles = 2 };
struct GPrim {
    float inv_model[16];
    float model[16];
    float lo[4], hi[4];  // box bounds or the triangle mesh's bounds (local); radius in lo[0] for spheres
    float color[4];
    float params[4];     // roughness, metal after material clamping
    uint32_t object, kind;
    uint32_t node_base, tri_base;  // kPrimTriangles: the mesh's hierarchy in the shared tables
};

// The primitive table and the shared triangle tables on one device.
struct PrimTable {
    const GPrim* prims;
    uint32_t n;
    const TriNode* nodes;
    const TriRec* tris;
};

}  // namespace irt

struct irt_workload {
    irt::Workload w;
};
