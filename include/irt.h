/*
 * irt.h — C-ABI of the B200 lighting hot path (ReSTIR direct + VPL indirect,
 * SDF soft-shadow visibility, SVGF) of the instantradiositytest renderer.
 *
 * The boundary replaces the wgpu binding contract of the reference's compute
 * passes:
 *   group 0 (scene)    common.wgsl:17-30,  src/renderer.rs:1185-1204
 *   group 1 (G-buffer) lighting.wgsl:1-5,  src/renderer.rs:1314-1324
 *   group 2 (per pass) lighting.wgsl:6-21, src/renderer.rs:1617-1674,
 *                      svgf.wgsl:8-17,     src/svgf.rs:163-211
 * and the pass schedule of Renderer::encode (src/renderer.rs:1873-1928) and
 * Svgf::encode (src/svgf.rs:140-261).
 *
 * Conventions: every call returns irt_status (0 = ok, negative = error) and
 * never throws; irt_last_error() gives the message of the last failure on a
 * context.  Device pointers are plain CUDA device addresses; `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).  No torch
 * types appear here.
 */
#ifndef IRT_H
#define IRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t irt_status;
#define IRT_OK 0
#define IRT_E_INVALID (-1)     /* bad argument / failed validation          */
#define IRT_E_CUDA (-2)        /* a CUDA runtime call failed                 */
#define IRT_E_ADMISSION (-3)   /* session would exceed the HBM budget        */
#define IRT_E_NOMEM (-4)       /* host allocation failed                     */
#define IRT_E_STATE (-5)       /* call made in the wrong order               */
#define IRT_E_DEVICE (-6)      /* a kernel reported a bounded-loop violation */
#define IRT_E_NODEVICE (-7)    /* no CUDA device is visible                  */

/* ---------------------------------------------------------------------------
 * Byte layouts shared with the caller.  Sizes are the reference's GPU struct
 * sizes (src/renderer.rs:2253-2261, common.wgsl:3-16); matrices are
 * column-major 4x4 f32 like glam::Mat4 and WGSL mat4x4<f32>.
 * ------------------------------------------------------------------------- */
typedef struct irt_mat4 { float m[16]; } irt_mat4;

/* common.wgsl:3-8, src/renderer.rs:52-66 — 384 bytes. */
typedef struct irt_frame {
    irt_mat4 vp, inv_vp, previous_vp, previous_inv_vp;
    float camera[4];
    uint32_t size[4];     /* width, height, frame_index, generation          */
    uint32_t counts[4];   /* lights, vpl_count, vpl_bounces, objects         */
    uint32_t restir[4];   /* direct cands, vpl cands, spatial nbrs, radius   */
    float temporal[4];    /* history weight, depth thr, normal thr, max hist */
    float sdf[4];         /* max steps, hit epsilon, soft-shadow k, 0        */
    float rr[4];          /* rr min, rr max, restir max history, 0           */
    uint32_t flags[4];    /* history enabled, previous generation, debug, 0  */
} irt_frame;

/* common.wgsl:9, src/renderer.rs:8-15 — 208 bytes.
 * info = [mesh id, material id, bits(uniform scale), bits(voxel diag*scale)] */
typedef struct irt_object {
    irt_mat4 model, previous, inverse;
    uint32_t info[4];
} irt_object;

/* common.wgsl:10, src/renderer.rs:16-28 — 128 bytes.
 * field = [atlas origin x,y,z, resolution]; grid = [1/spacing xyz, |spacing|];
 * geometry_lo.w = certified box flag; geometry_hi.w = 1/Lipschitz bound. */
typedef struct irt_mesh {
    float lo[4], hi[4];
    uint32_t geometry[4];
    uint32_t field[4];
    float grid[4];
    float geometry_lo[4], geometry_hi[4];
    float enclosing_sphere[4];
} irt_mesh;

/* common.wgsl:11, src/renderer.rs:29-36 — 64 bytes. */
typedef struct irt_material {
    float color[4], params[4];
    int32_t textures[4];
    uint32_t channels[4];
} irt_material;

/* common.wgsl:12, src/renderer.rs:37-43 — 48 bytes.
 * color_type.w > 0.5 marks a spot light. */
typedef struct irt_light {
    float position_strength[4], direction_angle[4], color_type[4];
} irt_light;

/* common.wgsl:13, src/scene.rs:136-143 — 64 bytes. */
typedef struct irt_vertex {
    float position[4], normal[4], tangent[4], uv[4];
} irt_vertex;

/* common.wgsl:14, src/renderer.rs:44-50 — 48 bytes.
 * info = [left|object, right, leaf flag, escape index] (preorder). */
typedef struct irt_node {
    float lo[4], hi[4];
    uint32_t info[4];
} irt_node;

/* common.wgsl:15 — 48 bytes. */
typedef struct irt_vpl {
    float position[4], normal[4], flux[4];
} irt_vpl;

/* common.wgsl:16 — 32 bytes; the device stores reservoirs in exactly this
 * layout (one 32-byte sector per pixel, read as two 128-bit vectors). */
typedef struct irt_reservoir {
    uint32_t id, source, count, age;
    float sum, selected_target, pdf;
    uint32_t generation;
} irt_reservoir;

/* settings.json / src/settings.rs:5-28. */
typedef struct irt_settings {
    uint32_t render_width, render_height;
    uint32_t vpl_count, vpl_max_bounces;
    float vpl_rr_min_survival, vpl_rr_max_survival;
    uint32_t restir_direct_candidates, restir_vpl_candidates;
    uint32_t restir_spatial_neighbors, restir_spatial_radius;
    uint32_t restir_max_history, svgf_iterations;
    float depth_threshold, normal_threshold, temporal_history_weight;
    uint32_t temporal_max_history;
    uint32_t sdf_max_steps;
    float sdf_hit_epsilon, sdf_soft_shadow_k, target_frame_ms;
} irt_settings;

/* Reference defaults (settings.json:1-22) with serde defaults for
 * restir_max_history / svgf_iterations (src/settings.rs:29-34). */
void irt_settings_default(irt_settings* out);
/* Same checks and messages as Settings::validate (src/settings.rs:42-105).
 * Writes the failing rule into msg (may be NULL). */
irt_status irt_settings_validate(const irt_settings* s, char* msg, size_t msg_len);

/* ---------------------------------------------------------------------------
 * Storage formats.
 * ------------------------------------------------------------------------- */
/* G-buffer planes (the reference's group-1 textures), all W*H row-major:
 *   F32:    depth f32, normal f32x4, color f32x4, params f32x2, motion f32x2
 *   F16:    depth f32, normal f16x4, color f16x4, params f16x2, motion f16x2
 *           (= the reference's Depth32Float / Rgba16Float / Rg16Float targets,
 *            src/renderer.rs:1207-1246)
 *   PACKED: depth f32, normal octahedral snorm16x2, color rgba8 unorm,
 *           params f16x2, motion f16x2                                        */
#define IRT_GBUFFER_F32 0
#define IRT_GBUFFER_F16 1
#define IRT_GBUFFER_PACKED 2

/* Radiance images (noisy lighting, SVGF temporal/scratch/feedback/output):
 *   F32: f32x4;  F16: f16x4 (the reference's Rgba16Float, src/svgf.rs:23). */
#define IRT_RADIANCE_F32 0
#define IRT_RADIANCE_F16 1

/* SVGF moments / history length:
 *   F32: f32x4 (m1, m2, age, 0) — the reference's Rgba32Float;
 *   F16: 8 bytes — f16 mean and f16 standard deviation of the luminance,
 *        then the history length as f32.  The second moment is stored
 *        central (a deviation, not E[x^2]), so HDR luminance^2 cannot
 *        overflow f16; the kernels combine moments in f32 with compensated
 *        (shifted / pooled-variance) forms of E[x^2] - E[x]^2.              */
#define IRT_MOMENTS_F32 0
#define IRT_MOMENTS_F16 1

/* SDF atlas texel format: F32 (R32Float, src/renderer.rs:820) or F16 with a
 * per-mesh scale (texel = f16(value / scale), scale in irt_mesh.lo[3]).      */
#define IRT_SDF_F32 0
#define IRT_SDF_F16 1

/* Which build of the library this is: "default", or "checked" for
 * libirt_checked.so, whose kernels test every index they take from data
 * (reservoir ids, reprojected and neighbouring pixels, ray-queue and output
 * slots, leaf-cache object ids) before following it and report a bad one as
 * IRT_E_DEVICE through irt_session_check instead of faulting.  No
 * counterpart in the reference (its shaders rely on robust buffer access). */
const char* irt_build_flavour(void);

/* ---------------------------------------------------------------------------
 * Context, scene, session.
 * ------------------------------------------------------------------------- */
typedef struct irt_context irt_context;
typedef struct irt_scene irt_scene;
typedef struct irt_session irt_session;

typedef struct irt_config {
    int32_t device;             /* CUDA ordinal                             */
    uint64_t hbm_budget_bytes;  /* 0 = 90% of the device's free memory      */
} irt_config;

irt_status irt_context_create(const irt_config* cfg, irt_context** out);
void irt_context_destroy(irt_context* ctx);
const char* irt_last_error(const irt_context* ctx);
/* Bytes of HBM the context's sessions and scenes hold right now. */
uint64_t irt_context_bytes_in_use(const irt_context* ctx);

/* Immutable scene data: mesh metadata and the SDF atlas (src/renderer.rs:
 * 776-888).  `atlas` is host memory of atlas_dims[0]*[1]*[2] texels, x
 * fastest, in `sdf_format`. */
irt_status irt_scene_create(irt_context* ctx, const irt_mesh* meshes, uint32_t mesh_count,
                            const void* atlas, const uint32_t atlas_dims[3], int32_t sdf_format,
                            irt_scene** out);
/* Per-frame scene data (src/renderer.rs:1738-1782): objects, preorder BVH
 * nodes (node_count must be 2*object_count-1) and lights, copied from host
 * memory on `stream`.  Validates every index the kernels follow. */
irt_status irt_scene_update(irt_scene* scene, const irt_object* objects, uint32_t object_count,
                            const irt_node* nodes, uint32_t node_count, const irt_light* lights,
                            uint32_t light_count, void* stream);
void irt_scene_destroy(irt_scene* scene);

/* Field sampler of a scene's SDF meshes.
 *   POINT:  sample_field of common.wgsl:31-38 — the cell's 8 texels loaded
 *           and weighted in f32 (the default; the reference's path when the
 *           adapter cannot filter R32Float).
 *   LINEAR: the reference's filtered variant, src/renderer.rs:277-286 (used
 *           there whenever FLOAT32_FILTERABLE is present,
 *           src/renderer.rs:736-739, :914-921, :1470-1471): one hardware
 *           linear fetch at (origin + q + .5) / atlas_dims (normalised;
 *           texel coordinate origin + q + .5) through a clamp-to-edge
 *           linear sampler.  The filter weights are the
 *           hardware's fixed-point ones (8 fractional bits), which the mesh
 *           bound's voxel/128 allowance covers (sdf.wgsl:16-17).
 * irt_scene_set_field_filter takes effect at the scene's next
 * irt_scene_update (which rebuilds the march's leaf-order cache under the
 * new sampler).  LINEAR needs an IRT_SDF_F32 atlas, as the reference's
 * filtered path does (R32Float): the texture unit filters 16-bit texels to a
 * 16-bit result, whose rounding exceeds the allowance away from surfaces;
 * IRT_E_INVALID for an F16 atlas. */
#define IRT_FIELD_POINT 0
#define IRT_FIELD_LINEAR 1
irt_status irt_scene_set_field_filter(irt_scene* scene, int32_t filter);
/* sample_field with `filter` of field mesh `mesh` at n grid-space points
 * q (device array of 3*n floats, q in [0, res-1]^3 as mesh_distance forms
 * it, sdf.wgsl:12); out: n floats on the device, dequantised (F16 atlases
 * times the mesh's scale).  The kernels' own sampler, exposed for parity
 * tests of the sampler alone (LINEAR is evaluated on F16 atlases too, to
 * measure the 16-bit filter); no counterpart in the reference. */
irt_status irt_scene_sample_field(const irt_scene* scene, int32_t filter, uint32_t mesh, const float* q,
                                  uint32_t n, float* out, void* stream);

typedef struct irt_session_desc {
    irt_settings settings;
    int32_t gbuffer_format;
    int32_t radiance_format;
    int32_t moments_format;
    int32_t fused;            /* schedule: 1 = candidates+temporal, spatial + ray set-up, persistent
                                 ray-queue march, resolve combine (default); 2 = candidates+temporal
                                 and spatial+resolve with the march inline per pixel; 0 = one kernel
                                 per reference entry point.  All three give identical results. */
    int32_t keep_candidates;  /* 1 = also write the candidates reservoirs [0] (parity/debug) */
    int32_t exact_march;      /* schedule 1: 1 = IEEE division and square root in the march
                                 (bit-identical to schedules 0 and 2); 0 = approximate (default) */
} irt_session_desc;

/* Allocates the session's persistent history (reservoirs, VPL archive, SVGF
 * targets, previous depth/normal).  Returns IRT_E_ADMISSION when the bytes
 * would exceed the context's HBM budget. */
irt_status irt_session_create(irt_context* ctx, const irt_session_desc* desc, irt_session** out);
/* HBM bytes a session with this description would hold. */
uint64_t irt_session_bytes(const irt_session_desc* desc);
void irt_session_destroy(irt_session* s);

typedef struct irt_gbuffer {
    int32_t format;           /* IRT_GBUFFER_*; must equal the session's     */
    const float* depth;       /* device pointers, W*H texels each            */
    const void* normal;
    const void* color;
    const void* params;
    const void* motion;
} irt_gbuffer;

/* The 8 lighting entry points of lighting.wgsl for one frame, in the order
 * of src/renderer.rs:1889-1928: VPL archive copy, candidates, temporal,
 * spatial, resolve.  current/previous VPL pools are caller-owned device
 * arrays of frame->counts[1] records. */
irt_status irt_frame_lighting(irt_session* s, const irt_scene* scene, const irt_frame* frame,
                              const irt_gbuffer* gbuffer, const irt_vpl* current_vpls,
                              const irt_vpl* previous_vpls, void* stream);
/* Svgf::encode (src/svgf.rs:140-261) followed by the depth/normal history
 * copy (src/renderer.rs:1951-1960). */
irt_status irt_frame_svgf(irt_session* s, const irt_frame* frame, const irt_gbuffer* gbuffer,
                          void* stream);
/* Both of the above. */
irt_status irt_render_frame(irt_session* s, const irt_scene* scene, const irt_frame* frame,
                            const irt_gbuffer* gbuffer, const irt_vpl* current_vpls,
                            const irt_vpl* previous_vpls, void* stream);

/* irt_render_frame from HOST inputs, pipelined: the G-buffer planes
 * (host_gbuffer holds host pointers, pinned for the copies to overlap) and
 * the VPL pool are copied into library-owned device staging (two G-buffer
 * slots, three VPL pools, created on the first call) on the session's own
 * copy stream while the previous frame still renders on `stream`; the frame
 * renders on `stream` once its inputs have landed, and, with out_host, its
 * filtered image (radiance format) is copied back to out_host on a second
 * copy stream — queued by the next call to run after that call's march, or
 * by irt_session_host_sync.  Call irt_session_host_sync before reading
 * out_host.  The
 * previous VPL pool of a call is the pool of the session's previous call
 * (zeros on the first).  No counterpart in the reference (its inputs are
 * GPU render targets). */
irt_status irt_render_frame_host(irt_session* s, const irt_scene* scene, const irt_frame* frame,
                                 const irt_gbuffer* host_gbuffer, const irt_vpl* host_vpls, void* out_host,
                                 void* stream);
/* The host copies (inputs consumed, outputs written) of every
 * irt_render_frame_host call so far: with stream == NULL the host waits for
 * them; otherwise work queued on `stream` afterwards waits for them. */
irt_status irt_session_host_sync(irt_session* s, void* stream);

#define IRT_BUF_DIRECT 0          /* f32x4: resolve_direct output            */
#define IRT_BUF_NOISY 1           /* radiance fmt: resolve_indirect output   */
#define IRT_BUF_FILTERED 2        /* radiance fmt: SVGF output of the frame  */
#define IRT_BUF_MOMENTS 3         /* moments fmt: moments written this frame */
#define IRT_BUF_RES_DIRECT 4      /* irt_reservoir[3][W*H] ([0],[1],[2])     */
#define IRT_BUF_RES_INDIRECT 5    /* irt_reservoir[3][W*H]                   */
#define IRT_BUF_VPL_ARCHIVE 6     /* irt_vpl[(max_history+1)*vpl_count]      */
#define IRT_BUF_PREV_DEPTH 7      /* f32                                     */
#define IRT_BUF_PREV_NORMAL 8     /* G-buffer normal format                  */
#define IRT_BUF_MOMENTS_OLD 9     /* moments slot the next frame reads       */
#define IRT_BUF_FEEDBACK 10       /* radiance fmt: a-trous-0 output (this)   */
#define IRT_BUF_FEEDBACK_OLD 11   /* radiance fmt: feedback the next frame reads */
#define IRT_BUF_ERROR 12          /* u32[4]: device error word (0 = none)    */
#define IRT_BUF_TEMPORAL 13       /* radiance fmt: svgf_temporal output      */
#define IRT_BUF_VARIANCE 14       /* radiance fmt: svgf_variance output      */
/* Device pointer and byte size of one session buffer.  "This frame" refers
 * to the last frame submitted. */
irt_status irt_session_buffer(irt_session* s, int32_t which, void** ptr, uint64_t* bytes);
/* Reservoir set k (0 = candidates, 1 = temporal, 2 = spatial/final) of a
 * domain (0 = direct, 1 = indirect): W*H irt_reservoir records.  Set 0 exists
 * only for unfused sessions or with keep_candidates. */
irt_status irt_session_reservoirs(irt_session* s, int32_t domain, int32_t k, void** ptr, uint64_t* bytes);
/* Reads and clears the device error word (bounded-loop violations); returns
 * IRT_E_DEVICE if a kernel reported one.  Synchronises `stream`. */
irt_status irt_session_check(irt_session* s, void* stream);
/* Device time of the last frame's passes (ms), measured with CUDA events
 * when profiling is on: names as in src/renderer.rs:2077-2092. */
irt_status irt_session_set_profiling(irt_session* s, int32_t on);
/* Ten values: archive copy, candidates+temporal, spatial (+ ray set-up),
 * march, resolve combine, SVGF temporal, SVGF variance, a-trous, history
 * copy, total.  Events are kept for the last 128 frames, so a timed run is
 * read back after it ends. */
irt_status irt_session_pass_ms(irt_session* s, float out_ms[10]);
irt_status irt_session_pass_ms_at(irt_session* s, uint32_t frame_index, float out_ms[10]);

/* SVGF spatial stages (variance bootstrap, then `iterations` a-trous passes)
 * of one frame for callers that cannot allocate device memory — a frame
 * thread that must not stall on an allocation, or a host that reserves all
 * device memory under its own allocator.  No counterpart in the reference
 * (there the filter's images are Svgf-owned textures).  The caller passes all
 * inputs — the svgf_temporal radiance (radiance_format) and moments
 * (moments_format: IRT_MOMENTS_F32 16-byte or IRT_MOMENTS_F16 8-byte texels),
 * e.g. a session's IRT_BUF_TEMPORAL and IRT_BUF_MOMENTS with that session's
 * formats — and outputs (filtered image; feedback image of the first pass,
 * may be NULL), in the radiance format given.  The frame's positions and
 * edge-stopping features and the two ping-pong images between passes live in
 * a fixed 20 MiB array of this library's device memory that every GPU loading
 * the library holds until exit; frames above 262144 pixels (512x512) are
 * rejected.  The first call on each device looks up that array's address
 * (with the device current), so it should come before any stream capture,
 * and the device must not be reset afterwards while the library is loaded.
 * All calls share the array: calls that overlap on the GPU race.  No
 * cudaMalloc/cudaFree is called.  With a session's inputs the outputs equal
 * the session's own filtered and feedback images bit for bit.  `err` (may be
 * NULL) receives a message on failure. */
irt_status irt_svgf_spatial_noalloc(const irt_frame* frame, const irt_gbuffer* gbuffer,
                                    int32_t radiance_format, int32_t moments_format, uint32_t iterations,
                                    const void* temporal_radiance, const void* moments,
                                    void* filtered_out, void* feedback_out, void* stream,
                                    char* err, size_t err_len);

/* ---------------------------------------------------------------------------
 * Host logic of src/renderer.rs used to build scene data (C++ equivalents).
 * ------------------------------------------------------------------------- */
/* is_box_geometry (src/renderer.rs:287-329). */
int32_t irt_is_box_geometry(const irt_vertex* vertices, uint32_t vertex_count,
                            const uint32_t* indices, uint32_t index_count,
                            const float lo[3], const float hi[3]);
/* field_lipschitz_bound (src/renderer.rs:330-358). */
float irt_field_lipschitz_bound(const float* samples, uint32_t resolution, const float spacing[3]);
/* Mesh metadata row of Renderer::new (src/renderer.rs:835-885): fills one
 * irt_mesh from geometry, SDF bounds and samples and its atlas origin. */
irt_status irt_mesh_metadata(const irt_vertex* vertices, uint32_t vertex_count,
                             const uint32_t* indices, uint32_t index_count, const float* samples,
                             uint32_t resolution, const float bounds_min[3],
                             const float bounds_max[3], const uint32_t atlas_origin[3],
                             irt_mesh* out);
/* Atlas tiling of Renderer::new (src/renderer.rs:778-795): tile grid and
 * extent for `count` meshes of max resolution `tile`. */
void irt_atlas_layout(uint32_t count, uint32_t tile, uint32_t grid_out[3], uint32_t extent_out[3]);
/* hierarchy() (src/renderer.rs:385-455): preorder median-split BVH over the
 * world AABBs of the objects' SDF bounds; writes 2*count-1 nodes. */
irt_status irt_build_hierarchy(const float* object_lo, const float* object_hi, uint32_t count,
                               irt_node* nodes_out);
/* objects() (src/renderer.rs:359-384) for one object. */
void irt_pack_object(const irt_mat4* model, const irt_mat4* previous, uint32_t mesh_id,
                     uint32_t material_id, const float sdf_lo[3], const float sdf_hi[3],
                     uint32_t sdf_resolution, irt_object* out);

/* ---------------------------------------------------------------------------
 * Synthetic workloads (seeded procedural rooms) and input producers: the
 * G-buffer producer that stands in for gbuffer.wgsl's raster and the VPL
 * generator that stands in for vpl.wgsl's ray queries.
 * ------------------------------------------------------------------------- */
typedef struct irt_workload_spec {
    uint64_t seed;
    uint32_t width, height;
    uint32_t n_boxes, n_spheres;
    int32_t room_single_mesh;     /* 1: the six wall slabs are one field mesh */
    uint32_t sdf_resolution;
    int32_t sdf_format;           /* IRT_SDF_*                                 */
    uint32_t n_lights;
    float radiance_lo, radiance_hi, emitter_size_lo, emitter_size_hi;
    uint32_t vpl_count, vpl_bounces;
    float orbit_deg_per_frame, dolly_m_per_frame;
} irt_workload_spec;

typedef struct irt_workload irt_workload;
/* Fills spec with config `which` (0: 256x160 room of 12 meshes, 64^3;
 * 1: 1920x1200 room of 24 meshes, 128^3, 8 emitters, 1024 VPLs). */
irt_status irt_workload_preset(int32_t which, irt_workload_spec* spec);
irt_status irt_workload_create(const irt_workload_spec* spec, irt_workload** out);
void irt_workload_destroy(irt_workload* wl);
uint32_t irt_workload_mesh_count(const irt_workload* wl);
uint32_t irt_workload_object_count(const irt_workload* wl);
uint32_t irt_workload_light_count(const irt_workload* wl);
const irt_mesh* irt_workload_meshes(const irt_workload* wl);
const void* irt_workload_atlas(const irt_workload* wl, uint32_t dims_out[3]);
int32_t irt_workload_sdf_format(const irt_workload* wl);
/* Settings of the workload (settings.json with the spec's size and VPLs). */
void irt_workload_settings(const irt_workload* wl, irt_settings* out);
/* Per-frame scene data and Frame uniform for frame `index` (camera path,
 * objects with previous transforms, BVH, lights), packed as in
 * Renderer::encode (src/renderer.rs:1687-1782).  `debug` is the debug mode. */
irt_status irt_workload_frame(irt_workload* wl, uint32_t index, uint32_t debug, irt_frame* frame,
                              irt_object* objects, irt_node* nodes, irt_light* lights);
/* CPU G-buffer producer (primary rays against the workload's analytic solids
 * or triangle hierarchies, back faces culled), writing the host planes of
 * `format` (see IRT_GBUFFER_*): depth, normal, color, params, motion. */
irt_status irt_workload_gbuffer_cpu(const irt_workload* wl, const irt_frame* frame,
                                    const irt_object* objects, int32_t format, float* depth,
                                    void* normal, void* color, void* params, void* motion);
/* Scene-format loader: Scene::load + Scene::validate (src/scene.rs:157-382)
 * of the version-1 manifest at `manifest_path` and the binaries it names
 * (paths relative to the manifest's directory): meshes as triangle lists
 * (64-byte vertices, u32 indices) with their SDF fields (res^3 f32), objects,
 * materials, lights and the fixed camera.  The workload's atlas, mesh rows,
 * per-frame data and producers then serve the file's scene (triangle casts;
 * textured materials are rejected).  From `spec` only width, height,
 * sdf_format, vpl_count and vpl_bounces are used.  On failure returns
 * IRT_E_INVALID (or IRT_E_NOMEM) and writes the reason, prefixed as the
 * reference's error context ("reading <path>", "parsing <path>",
 * "scene <path>", "mesh <id>"), NUL-terminated into error[0..error_len). */
irt_status irt_workload_load(const char* manifest_path, const irt_workload_spec* spec,
                             irt_workload** out, char* error, uint64_t error_len);
/* CPU VPL generator: vpl.wgsl:1-47 with ray casts against the workload's
 * analytic solids or triangle hierarchies. */
irt_status irt_workload_vpls_cpu(const irt_workload* wl, const irt_frame* frame,
                                 const irt_object* objects, const irt_light* lights,
                                 irt_vpl* out);
/* CUDA G-buffer producer: same contract as the CPU one, device planes. */
irt_status irt_gbuffer_render(irt_context* ctx, const irt_workload* wl, const irt_frame* frame,
                              const irt_object* objects, int32_t format, float* depth,
                              void* normal, void* color, void* params, void* motion,
                              void* stream);
/* CUDA VPL generator (replaces the vpl.wgsl compute pass, vpl.wgsl:1-47, and
 * its dispatch in src/renderer.rs:1873-1884): frame->counts[1] paths of up to
 * frame->counts[2] bounces from the lights last uploaded to `scene`
 * (irt_scene_update), written to the device pool `out`.  Ray casts run
 * against the workload's primitives: analytic solids or the triangle
 * hierarchies of a loaded scene (the reference uses a hardware ray query
 * against its TLAS).  Same contract as irt_workload_vpls_cpu. */
irt_status irt_vpl_generate(irt_scene* scene, const irt_workload* wl, const irt_frame* frame,
                            irt_vpl* out, void* stream);

/* Presentation pass (present.wgsl:1-8 drawn into the Rgba8UnormSrgb display
 * target, src/renderer.rs:1300-1306, :1961): each pixel of a radiance image
 * (IRT_RADIANCE_* format, e.g. IRT_BUF_FILTERED), clamped to [0, 1],
 * sRGB-encoded and rounded to 8 bits, alpha 255; rgba8 is a device buffer of
 * width*height*4 bytes.  Capture to PNG (src/renderer.rs:2109-2163) is the
 * host's: read rgba8 back and encode it (instantradiositytest_b200.present). */
irt_status irt_present(const void* radiance, int32_t radiance_format, uint32_t width, uint32_t height,
                       uint8_t* rgba8, void* stream);

/* ---------------------------------------------------------------------------
 * Batched views (no counterpart in the reference, which renders one view per
 * Renderer).  A batch renders many views of uneven size — each a session of
 * its own with its own history, over its own scene or one shared with other
 * views — with ONE launch per pass for all of them: per pass a tile table
 * maps blocks to (view, tile) and per-view argument tables live on the
 * device; the march is one persistent launch whose CTAs stage each scene's
 * compact records in shared memory once and consume every view's ray queue
 * of that scene.  With use_graphs, each frame's launches (frame upload
 * included) are captured once per frame parity as a CUDA graph and replayed.
 * Tile shapes come from the batch's autotuner (irt_batch_autotune).  Every
 * view's results are those of irt_render_frame on that view alone.
 * All views of a batch render the same frame index each call; debug views
 * (frame.flags[2] != 0) are not batched.
 * ------------------------------------------------------------------------- */
typedef struct irt_batch irt_batch;

typedef struct irt_batch_desc {
    irt_settings settings;      /* shared by all views; render_width/height ignored */
    int32_t gbuffer_format, radiance_format, moments_format;
    int32_t use_graphs;         /* 1 = capture and replay a CUDA graph per frame     */
    uint32_t n_views;
    const uint32_t* widths;     /* n_views entries                                   */
    const uint32_t* heights;    /* n_views entries                                   */
    const uint32_t* vpl_counts; /* n_views entries, or NULL = settings.vpl_count     */
} irt_batch_desc;

irt_status irt_batch_create(irt_context* ctx, const irt_batch_desc* desc, irt_batch** out);
/* One frame of every view: scenes[v] (already updated for this frame with
 * irt_scene_update on the same stream), frames[v], gbuffers[v], current and
 * previous VPL pools of view v.  The batch runs on a stream of its own that
 * waits for `stream` and that `stream` then waits for. */
irt_status irt_batch_render(irt_batch* b, irt_scene* const* scenes, const irt_frame* frames,
                            const irt_gbuffer* gbuffers, const irt_vpl* const* current,
                            const irt_vpl* const* previous, void* stream);
/* The session that holds view v's history and outputs (irt_session_buffer). */
irt_session* irt_batch_view(irt_batch* b, uint32_t view);
/* The next max(frames, 5) calls of irt_batch_render try the candidate tile
 * shapes (2-D kernels: 32x8, 64x4, 16x16, 128x2, 256x1; march CTAs per SM)
 * on one wave and time every pass, each pass keeping its fastest shape; the
 * 5 calls after them time the frame at each wave budget and keep the
 * fastest. */
irt_status irt_batch_autotune(irt_batch* b, uint32_t frames);
/* Views run in waves: consecutive views whose pixels add up to at most
 * budget_px share one launch per pass, wave after wave, so a wave's buffers
 * stay in L2 between its passes (0 = all views in one wave).  The autotuner
 * also picks it, among 0, 8, 4, 2 and 1 Mi pixels. */
irt_status irt_batch_set_waves(irt_batch* b, uint64_t budget_px);
/* The tile shapes and waves in use, as text
 * ("reuse=32x8 ... march_ctas_per_sm=max waves=3 wave_budget_px=4194304"). */
irt_status irt_batch_tuning(const irt_batch* b, char* out, size_t len);
/* Device time of the last directly launched frame's passes (ms), 12 values:
 * guides, archive, reuse, spatial, march, combine, temporal, variance,
 * a-trous (all iterations), history, total, and 1 if the last frame was a
 * graph replay (0 otherwise). */
irt_status irt_batch_pass_ms(irt_batch* b, float* out12);
void irt_batch_destroy(irt_batch* b);

/* ---------------------------------------------------------------------------
 * Render server: continuous batching of render sessions (no counterpart in
 * the reference, which renders one view from one Renderer).
 *
 * Requests arrive over time (arrival_s, seconds after irt_server_run starts);
 * each is a render session of `frames` frames over a synthetic workload (its
 * scene, camera path and frame size).  The server admits waiting requests in
 * arrival order while their HBM bytes (session history, scene, per-frame
 * inputs) fit the server's budget and a slot is free; an admitted session
 * keeps its reservoirs and SVGF history resident until its last frame and
 * then frees them, so the next request can enter.  Admitted sessions are
 * spread over CUDA streams and their frames interleave on the device: each
 * frame is scene update, G-buffer, VPL generation and the lighting + SVGF
 * hot path (irt_render_frame) on the session's stream.  Frames of a session
 * are paced at frame_rate (0 = as fast as possible) with at most two in
 * flight.  A session's results do not depend on what else runs with it.
 * ------------------------------------------------------------------------- */
typedef struct irt_server irt_server;

typedef struct irt_server_desc {
    uint64_t hbm_budget_bytes;  /* admission budget for all admitted sessions   */
    uint32_t max_sessions;      /* admitted at once (0 = limited by bytes only) */
    uint32_t streams;           /* CUDA streams sessions are spread over (>= 1) */
    float frame_rate;           /* per-session pacing in frames/s; 0 = none     */
    int32_t gbuffer_format, radiance_format, moments_format;
    int32_t fused;              /* session schedule (irt_session_desc.fused)    */
} irt_server_desc;

typedef struct irt_request {
    uint64_t id;
    double arrival_s;           /* seconds after irt_server_run starts          */
    uint32_t frames;
    irt_workload* workload;     /* scene + camera path; caller-owned, outlives the run */
    uint32_t capture_frame;     /* frame whose filtered image is copied ...     */
    void* capture;              /* ... to this host buffer (NULL = none)        */
    double* times;              /* NULL, or 3 doubles written by irt_server_run:
                                   admitted, last frame done, retired (seconds
                                   after the run starts; -1 if never admitted) */
} irt_request;

typedef struct irt_server_stats {
    uint64_t frames, sessions, rejected;
    double pixel_frames;        /* sum of W*H over rendered frames              */
    double seconds;             /* first admission to last completion           */
    double mpix_frames_per_s;
    float p50_latency_ms, p99_latency_ms;  /* frame due -> frame done            */
    float p50_frame_ms, p99_frame_ms;      /* device time of a frame, start->end */
    float p50_wait_ms, p99_wait_ms;        /* arrival -> admission               */
    float mean_active, peak_active;
    uint64_t peak_bytes;
} irt_server_stats;

irt_status irt_server_create(irt_context* ctx, const irt_server_desc* desc, irt_server** out);
/* Queues a request (before or between runs).  A request whose bytes exceed
 * the whole budget is rejected at run time and counted in stats.rejected. */
irt_status irt_server_submit(irt_server* server, const irt_request* request);
/* Serves every queued request to completion; host-blocking. */
irt_status irt_server_run(irt_server* server, irt_server_stats* stats);
/* HBM bytes the server charges a request against its budget. */
uint64_t irt_server_request_bytes(const irt_server* server, const irt_request* request);
void irt_server_destroy(irt_server* server);

#ifdef __cplusplus
}
#endif
#endif /* IRT_H */
