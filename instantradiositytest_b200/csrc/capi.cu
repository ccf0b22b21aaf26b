// capi.cu — the irt_* C-ABI: context, scene and session objects and the
// per-frame pass schedule of Renderer::encode (src/renderer.rs:1873-1960) and
// Svgf::encode (src/svgf.rs:140-261).  No exception crosses the boundary.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "workload.h"


extern "C" {

// ------------------------------------------------------------------ context
irt_status irt_context_create(const irt_config* cfg, irt_context** out) {
    if (!out) return IRT_E_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return IRT_E_NODEVICE;
    }
    int dev = cfg ? cfg->device : 0;
    if (dev < 0 || dev >= count) return IRT_E_INVALID;
    irt_context* ctx = new (std::nothrow) irt_context();
    if (!ctx) return IRT_E_NOMEM;
    ctx->device = dev;
    DeviceGuard g(dev);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        delete ctx;
        return IRT_E_CUDA;
    }
    ctx->budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (uint64_t)(free_b * 0.9);
    *out = ctx;
    return IRT_OK;
}

void irt_context_destroy(irt_context* ctx) { delete ctx; }

const char* irt_last_error(const irt_context* ctx) {
    if (!ctx) return "null context";
    std::lock_guard<std::mutex> g(ctx->mu);
    return ctx->last_error.c_str();
}

uint64_t irt_context_bytes_in_use(const irt_context* ctx) { return ctx ? ctx->in_use.load() : 0; }

// ------------------------------------------------------------------ scene
irt_status irt_scene_create(irt_context* ctx, const irt_mesh* meshes, uint32_t mesh_count, const void* atlas,
                            const uint32_t atlas_dims[3], int32_t sdf_format, irt_scene** out) {
    if (!ctx || !out || !meshes || mesh_count == 0 || !atlas || !atlas_dims) return IRT_E_INVALID;
    if (sdf_format != IRT_SDF_F32 && sdf_format != IRT_SDF_F16) return IRT_E_INVALID;
    *out = nullptr;
    // Every texel a mesh can address must lie inside the atlas.
    for (uint32_t m = 0; m < mesh_count; m++) {
        const irt_mesh& me = meshes[m];
        if (me.geometry_lo[3] > .5f) continue;
        uint32_t res = me.field[3];
        if (res < 2) {
            ctx->set_error("mesh resolution below 2");
            return IRT_E_INVALID;
        }
        for (int a = 0; a < 3; a++)
            if ((uint64_t)me.field[a] + res > atlas_dims[a]) {
                ctx->set_error("mesh field tile outside the atlas");
                return IRT_E_INVALID;
            }
    }
    DeviceGuard g(ctx->device);
    irt_scene* sc = new (std::nothrow) irt_scene();
    if (!sc) return IRT_E_NOMEM;
    sc->ctx = ctx;
    sc->mesh_count = mesh_count;
    sc->sdf_f16 = sdf_format == IRT_SDF_F16;
    for (int a = 0; a < 3; a++) sc->atlas_dims[a] = atlas_dims[a];
    sc->host_meshes.assign(meshes, meshes + mesh_count);
    auto fail = [&](irt_status s) {
        irt_scene_destroy(sc);
        return s;
    };
    irt_status st = dev_alloc(ctx, &sc->meshes, sizeof(irt_mesh) * mesh_count, sc->bytes);
    if (st) return fail(st);
    cudaError_t e = cudaMemcpy(sc->meshes, meshes, sizeof(irt_mesh) * mesh_count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "mesh upload"));
    cudaChannelFormatDesc cd =
        sdf_format == IRT_SDF_F16 ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
    cudaExtent ext = make_cudaExtent(atlas_dims[0], atlas_dims[1], atlas_dims[2]);
    e = cudaMalloc3DArray(&sc->atlas_array, &cd, ext);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "cudaMalloc3DArray"));
    size_t texel = sdf_format == IRT_SDF_F16 ? 2 : 4;
    sc->bytes += texel * atlas_dims[0] * atlas_dims[1] * (size_t)atlas_dims[2];
    cudaMemcpy3DParms cp{};
    cp.srcPtr = make_cudaPitchedPtr(const_cast<void*>(atlas), atlas_dims[0] * texel, atlas_dims[0], atlas_dims[1]);
    cp.dstArray = sc->atlas_array;
    cp.extent = ext;
    cp.kind = cudaMemcpyHostToDevice;
    e = cudaMemcpy3D(&cp);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "atlas upload"));
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = sc->atlas_array;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&sc->atlas, &rd, &td, nullptr);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "texture object"));
    // The reference's field_sampler (src/renderer.rs:914-921): linear
    // min/mag filter, clamp-to-edge.  It samples at the normalised
    // coordinate (origin + q + .5) / dims; this sampler takes the same point
    // as the texel coordinate origin + q + .5, without the division.
    td.filterMode = cudaFilterModeLinear;
    td.normalizedCoords = 0;
    e = cudaCreateTextureObject(&sc->atlas_linear, &rd, &td, nullptr);
    if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "linear texture object"));
    // Corner cells of the field meshes (DevScene::sdf_cells); a mesh's first
    // record index goes into hi[3] of its rows, which nothing else reads.
    {
        uint64_t total = 0;
        std::vector<uint64_t> base(mesh_count, 0);
        for (uint32_t m = 0; m < mesh_count; m++) {
            if (meshes[m].geometry_lo[3] > .5f) continue;
            const uint64_t n = meshes[m].field[3] - 1u;
            base[m] = total;
            total += n * n * n;
        }
        if (total > 0xffffffffull) {
            ctx->set_error("field meshes exceed 2^32 SDF cells");
            return fail(IRT_E_INVALID);
        }
        if (total > 0) {
            st = dev_alloc(ctx, &sc->sdf_cells, total * (sc->sdf_f16 ? 16 : 32), sc->bytes);
            if (st) return fail(st);
            for (uint32_t m = 0; m < mesh_count; m++) {
                if (meshes[m].geometry_lo[3] > .5f) continue;
                e = irt_pack_sdf_cells(sc->atlas, sc->sdf_f16, meshes[m].field, meshes[m].field[3], base[m],
                                       sc->sdf_cells, nullptr);
                if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "corner cells"));
                const uint32_t b32 = (uint32_t)base[m];
                std::memcpy(&sc->host_meshes[m].hi[3], &b32, 4);
            }
            e = cudaStreamSynchronize(nullptr);
            if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "corner cells"));
            e = cudaMemcpy(sc->meshes, sc->host_meshes.data(), sizeof(irt_mesh) * mesh_count, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return fail(cuda_fail(ctx, e, "mesh upload"));
        }
    }
    ctx->in_use += sc->bytes;
    *out = sc;
    return IRT_OK;
}

irt_status irt_scene_update(irt_scene* sc, const irt_object* objects, uint32_t object_count, const irt_node* nodes,
                            uint32_t node_count, const irt_light* lights, uint32_t light_count, void* stream) {
    if (!sc) return IRT_E_INVALID;
    irt_context* ctx = sc->ctx;
    if (!objects || object_count == 0 || !nodes || node_count != 2 * object_count - 1 || (light_count && !lights)) {
        ctx->set_error("scene update needs objects and 2N-1 nodes");
        return IRT_E_INVALID;
    }
    if (object_count > kMaxMarchObjects) {
        ctx->set_error("more objects than the march scene holds (1024)");
        return IRT_E_INVALID;
    }
    // Validate every index the device walk follows: mesh ids, leaf object
    // ids, and escape links that strictly advance and stay within 2N-1.
    for (uint32_t i = 0; i < object_count; i++)
        if (objects[i].info[0] >= sc->mesh_count) {
            ctx->set_error("object references a mesh outside the scene");
            return IRT_E_INVALID;
        }
    for (uint32_t i = 0; i < node_count; i++) {
        const irt_node& n = nodes[i];
        if (n.info[3] <= i || n.info[3] > node_count || (n.info[2] == 1u && n.info[0] >= object_count)) {
            ctx->set_error("malformed BVH node");
            return IRT_E_INVALID;
        }
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (object_count > sc->object_cap) {
        uint64_t before = sc->bytes;
        if (sc->objects) cudaFree(sc->objects);
        if (sc->nodes) cudaFree(sc->nodes);
        sc->objects = nullptr;
        sc->nodes = nullptr;
        uint64_t added = 0;
        irt_status s1 = dev_alloc(ctx, &sc->objects, sizeof(irt_object) * object_count, added);
        if (s1) return s1;
        s1 = dev_alloc(ctx, &sc->nodes, sizeof(irt_node) * (2 * (size_t)object_count - 1), added);
        if (s1) return s1;
        sc->object_cap = object_count;
        sc->bytes = before + added;
        ctx->in_use += added;
    }
    if (light_count > sc->light_cap) {
        if (sc->lights) cudaFree(sc->lights);
        if (sc->lights_prep) cudaFree(sc->lights_prep);
        sc->lights = nullptr;
        sc->lights_prep = nullptr;
        uint64_t added = 0;
        irt_status s1 = dev_alloc(ctx, &sc->lights, sizeof(irt_light) * light_count, added);
        if (s1) return s1;
        s1 = dev_alloc(ctx, &sc->lights_prep, sizeof(irt_light) * light_count, added);
        if (s1) return s1;
        sc->light_cap = light_count;
        sc->bytes += added;
        ctx->in_use += added;
    }
    // Per-frame data goes through a pinned staging slot: the copies are then
    // truly asynchronous (a copy from pageable memory can hold the host until
    // the stream drains), and the slot is reused only after its copies ran.
    const size_t ob = sizeof(irt_object) * object_count, nb = sizeof(irt_node) * node_count,
                 lb = sizeof(irt_light) * light_count;
    const uint32_t mbytes_up = irt_march_scene_bytes(object_count);
    const size_t need = ob + nb + lb + mbytes_up + 64;
    const int slot = (int)(sc->updates % 2u);
    if (!sc->pinned_free[slot]) CK(cudaEventCreateWithFlags(&sc->pinned_free[slot], cudaEventDisableTiming), "staging");
    CK(cudaEventSynchronize(sc->pinned_free[slot]), "staging");
    if (sc->pinned_cap[slot] < need) {
        if (sc->pinned[slot]) cudaFreeHost(sc->pinned[slot]);
        sc->pinned[slot] = nullptr;
        sc->pinned_cap[slot] = 0;
        CK(cudaMallocHost(&sc->pinned[slot], need), "staging");
        sc->pinned_cap[slot] = need;
    }
    unsigned char* stage = sc->pinned[slot];
    std::memcpy(stage, objects, ob);
    std::memcpy(stage + ob, nodes, nb);
    if (lb) std::memcpy(stage + ob + nb, lights, lb);
    unsigned char* stage_march = stage + ((ob + nb + lb + 15) & ~size_t(15));
    CK(cudaMemcpyAsync(sc->objects, stage, ob, cudaMemcpyHostToDevice, st), "objects");
    CK(cudaMemcpyAsync(sc->nodes, stage + ob, nb, cudaMemcpyHostToDevice, st), "nodes");
    if (light_count) {
        CK(cudaMemcpyAsync(sc->lights, stage + ob + nb, lb, cudaMemcpyHostToDevice, st), "lights");
        CK(irt_launch_prepare_lights(sc->lights, light_count, sc->lights_prep, st), "light preparation");
    }
    // Compact march scene: the same values, laid out for shared memory.
    const uint32_t mbytes = irt_march_scene_bytes(object_count);
    if (sc->march_host.size() * 16 < mbytes) {
        if (sc->march_scene) cudaFree(sc->march_scene);
        sc->march_scene = nullptr;
        uint64_t added = 0;
        irt_status s1 = dev_alloc(ctx, &sc->march_scene, mbytes, added);
        if (s1) return s1;
        sc->bytes += added;
        ctx->in_use += added;
    }
    sc->march_host.assign(mbytes / 16, make_float4(0.f, 0.f, 0.f, 0.f));
    irtd::MNode* mn = reinterpret_cast<irtd::MNode*>(sc->march_host.data());
    irtd::MObj* mo = reinterpret_cast<irtd::MObj*>(mn + node_count);
    auto bits = [](uint32_t u) {
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    };
    std::vector<uint32_t> leaf_of(object_count, 0);
    for (uint32_t i = 0; i < node_count; i++) {
        const irt_node& n = nodes[i];
        mn[i].a = make_float4(n.lo[0], n.lo[1], n.lo[2], bits(n.info[3]));
        mn[i].b = make_float4(n.hi[0], n.hi[1], n.hi[2], bits(n.info[2] == 1u ? n.info[0] : 0xffffffffu));
        if (n.info[2] == 1u) leaf_of[n.info[0]] = i;
    }
    for (uint32_t i = 0; i < object_count; i++) {
        const irt_object& o = objects[i];
        const irt_mesh& m = sc->host_meshes[o.info[0]];
        const float* inv = o.inverse.m;  // column-major
        mo[i].rx = make_float4(inv[0], inv[4], inv[8], inv[12]);
        mo[i].ry = make_float4(inv[1], inv[5], inv[9], inv[13]);
        mo[i].rz = make_float4(inv[2], inv[6], inv[10], inv[14]);
        mo[i].meta = make_float4(bits(o.info[2]), bits(o.info[3]), bits(o.info[0]), bits(leaf_of[i]));
        mo[i].lo = make_float4(m.lo[0], m.lo[1], m.lo[2], m.lo[3]);
        mo[i].hi = make_float4(m.hi[0], m.hi[1], m.hi[2], m.hi[3]);
        mo[i].field = make_uint4(m.field[0], m.field[1], m.field[2], m.field[3]);
        mo[i].grid = make_float4(m.grid[0], m.grid[1], m.grid[2], m.grid[3]);
        mo[i].glo = make_float4(m.geometry_lo[0], m.geometry_lo[1], m.geometry_lo[2], m.geometry_lo[3]);
        mo[i].ghi = make_float4(m.geometry_hi[0], m.geometry_hi[1], m.geometry_hi[2], m.geometry_hi[3]);
        mo[i].sphere = make_float4(m.enclosing_sphere[0], m.enclosing_sphere[1], m.enclosing_sphere[2],
                                   m.enclosing_sphere[3]);
    }
    std::memcpy(stage_march, sc->march_host.data(), mbytes);
    CK(cudaMemcpyAsync(sc->march_scene, stage_march, mbytes, cudaMemcpyHostToDevice, st), "march scene");
    CK(cudaEventRecord(sc->pinned_free[slot], st), "staging");
    sc->updates++;
    // A new field sampler changes every object distance the leaf-order cache
    // bounds, so it takes effect here, with the cache rebuilt.
    if (sc->field_linear != sc->field_linear_requested) {
        sc->field_linear = sc->field_linear_requested;
        sc->cached_nodes.clear();
        sc->cached_objects.clear();
    }
    // Leaf-order cache, rebuilt on the device when the BVH or an object
    // changes (static scenes build it once).
    if (sc->cached_nodes.size() != node_count || sc->cached_objects.size() != object_count ||
        std::memcmp(sc->cached_nodes.data(), nodes, sizeof(irt_node) * node_count) != 0 ||
        std::memcmp(sc->cached_objects.data(), objects, sizeof(irt_object) * object_count) != 0) {
        const size_t words = (size_t)kGridRes * kGridRes * kGridRes * kCellWords;
        if (!sc->cells) {
            uint64_t added = 0;
            irt_status s1 = dev_alloc(ctx, &sc->cells, words * 4, added);
            if (s1) return s1;
            sc->bytes += added;
            ctx->in_use += added;
        }
        const uint32_t R = kGridRes + 1;
        const size_t corner_floats = (size_t)R * R * R * object_count;
        if (object_count <= kMaxCornerObjects && sc->corner_cap < corner_floats) {
            if (sc->corners) cudaFree(sc->corners);
            sc->corners = nullptr;
            uint64_t added = 0;
            irt_status s1 = dev_alloc(ctx, &sc->corners, corner_floats * 4, added);
            if (s1) return s1;
            sc->corner_cap = corner_floats;
            sc->bytes += added;
            ctx->in_use += added;
        }
        LeafCacheLaunch LC{};
        LC.march_scene = sc->march_scene;
        LC.n = object_count;
        LC.atlas = sc->atlas;
        LC.sdf_f16 = sc->sdf_f16;
        LC.sdf_cells = sc->sdf_cells;
        LC.field_filter = scene_field_filter(sc);
        for (int a = 0; a < 3; a++) {
            // The grid covers the root box grown by 0.1 % and 1 mm.
            double ext = (double)nodes[0].hi[a] - (double)nodes[0].lo[a];
            double lo = (double)nodes[0].lo[a] - 1e-3 * ext - 1e-3;
            double hi = (double)nodes[0].hi[a] + 1e-3 * ext + 1e-3;
            LC.grid_org_d[a] = lo;
            LC.grid_size_d[a] = (hi - lo) / kGridRes;
            sc->grid_org[a] = (float)lo;
            sc->grid_inv[a] = (float)(kGridRes / (hi - lo));
        }
        LC.corners = object_count <= kMaxCornerObjects ? sc->corners : nullptr;
        LC.cells = reinterpret_cast<uint32_t*>(sc->cells);
        CK(irt_launch_leaf_cache(LC, st), "leaf cache");
        sc->cached_nodes.assign(nodes, nodes + node_count);
        sc->cached_objects.assign(objects, objects + object_count);
    }
    sc->object_count = object_count;
    sc->light_count = light_count;
    return IRT_OK;
}

irt_status irt_vpl_generate(irt_scene* sc, const irt_workload* wl, const irt_frame* f, irt_vpl* out, void* stream) {
    if (!sc || !wl || !f || !out) return IRT_E_INVALID;
    irt_context* ctx = sc->ctx;
    if (f->counts[0] > sc->light_count || (f->counts[0] && !sc->lights)) {
        ctx->set_error("frame light count exceeds the scene's uploaded lights");
        return IRT_E_INVALID;
    }
    if (f->counts[2] > 64) {
        ctx->set_error("VPL bounce count out of range");
        return IRT_E_INVALID;
    }
    DeviceGuard dg(ctx->device);
    VplLaunch V{};
    V.frame = f;
    V.lights = sc->lights;
    V.out = out;
    CK(irt_workload_prims(wl, &V.prims), "workload primitives");
    CK(irt_launch_vpls(V, static_cast<cudaStream_t>(stream)), "vpl kernel");
    return IRT_OK;
}

const char* irt_build_flavour(void) { return IRT_CHECKED ? "checked" : "default"; }

irt_status irt_scene_set_field_filter(irt_scene* sc, int32_t filter) {
    if (!sc) return IRT_E_INVALID;
    if (filter != IRT_FIELD_POINT && filter != IRT_FIELD_LINEAR) {
        sc->ctx->set_error("unknown field filter");
        return IRT_E_INVALID;
    }
    if (filter == IRT_FIELD_LINEAR && sc->sdf_f16) {
        // The texture unit filters 16-bit texels to a 16-bit result: away
        // from surfaces the rounding exceeds the bound's voxel/128 allowance.
        // The reference filters R32Float fields only.
        sc->ctx->set_error("the filtered field sampler needs an f32 SDF atlas (16-bit texels filter to 16-bit values)");
        return IRT_E_INVALID;
    }
    sc->field_linear_requested = filter == IRT_FIELD_LINEAR;
    return IRT_OK;
}

irt_status irt_scene_sample_field(const irt_scene* sc, int32_t filter, uint32_t mesh, const float* q, uint32_t n,
                                  float* out, void* stream) {
    if (!sc) return IRT_E_INVALID;
    irt_context* ctx = sc->ctx;
    if ((filter != IRT_FIELD_POINT && filter != IRT_FIELD_LINEAR) || mesh >= sc->mesh_count || !q || !out || !n) {
        ctx->set_error("sample_field: bad filter, mesh index, points or output");
        return IRT_E_INVALID;
    }
    const irt_mesh& row = sc->host_meshes[mesh];
    if (row.geometry_lo[3] > .5f) {
        ctx->set_error("sample_field: the mesh is a certified box and has no field");
        return IRT_E_INVALID;
    }
    DeviceGuard dg(ctx->device);
    irtd::DevScene d{};
    d.atlas = sc->atlas;
    d.sdf_f16 = sc->sdf_f16;
    d.sdf_cells = sc->sdf_cells;
    d.filter = scene_field_filter(sc);
    d.filter.linear = filter == IRT_FIELD_LINEAR ? sc->atlas_linear : 0;
    CK(irt_launch_sample_field(d, row, q, n, out, static_cast<cudaStream_t>(stream)), "sample_field kernel");
    return IRT_OK;
}

void irt_scene_destroy(irt_scene* sc) {
    if (!sc) return;
    DeviceGuard g(sc->ctx->device);
    if (sc->atlas) cudaDestroyTextureObject(sc->atlas);
    if (sc->atlas_linear) cudaDestroyTextureObject(sc->atlas_linear);
    if (sc->atlas_array) cudaFreeArray(sc->atlas_array);
    if (sc->sdf_cells) cudaFree(sc->sdf_cells);
    if (sc->meshes) cudaFree(sc->meshes);
    if (sc->objects) cudaFree(sc->objects);
    if (sc->nodes) cudaFree(sc->nodes);
    if (sc->lights) cudaFree(sc->lights);
    if (sc->lights_prep) cudaFree(sc->lights_prep);
    if (sc->march_scene) cudaFree(sc->march_scene);
    if (sc->cells) cudaFree(sc->cells);
    if (sc->corners) cudaFree(sc->corners);
    for (int k = 0; k < 2; k++) {
        if (sc->pinned_free[k]) {
            cudaEventSynchronize(sc->pinned_free[k]);
            cudaEventDestroy(sc->pinned_free[k]);
        }
        if (sc->pinned[k]) cudaFreeHost(sc->pinned[k]);
    }
    if (sc->ctx->in_use >= sc->bytes) sc->ctx->in_use -= sc->bytes;
    delete sc;
}

// ------------------------------------------------------------------ session
uint64_t irt_session_bytes(const irt_session_desc* d) {
    if (!d) return 0;
    uint64_t P = (uint64_t)d->settings.render_width * d->settings.render_height;
    uint64_t rad = d->radiance_format == IRT_RADIANCE_F16 ? 8 : 16;
    uint64_t res_sets = needs_candidates(*d) ? 3 : 2;
    uint64_t b = 0;
    b += 2 * res_sets * P * 32;                                                     // reservoirs
    b += (uint64_t)(d->settings.restir_max_history + 1) * d->settings.vpl_count * 48;  // archive
    b += P * 4 + P * normal_bytes_of(d->gbuffer_format);                            // previous depth/normal
    b += P * 16;                                                                    // direct f32x4
    b += P * rad * 7;  // noisy, feedback x2, temporal, scratch x2, filtered
    b += P * (d->moments_format == IRT_MOMENTS_F16 ? 8 : 16) * 2;  // moments x2
    b += 16;           // error word
    if (d->fused == 1) b += P * (2 * sizeof(RayRecord) + 2 * 4 + 2 * 16) + 16;  // ray queue, vis, pending
    b += P * 16 * 2;                                                             // position guides
    b += P * 32;                                                                 // SVGF features
    return b;
}

irt_status irt_session_create(irt_context* ctx, const irt_session_desc* desc, irt_session** out) {
    if (!ctx || !desc || !out) return IRT_E_INVALID;
    *out = nullptr;
    char msg[128];
    if (irt_settings_validate(&desc->settings, msg, sizeof(msg)) != IRT_OK) {
        ctx->set_error(msg);
        return IRT_E_INVALID;
    }
    if (desc->gbuffer_format < IRT_GBUFFER_F32 || desc->gbuffer_format > IRT_GBUFFER_PACKED ||
        (desc->radiance_format != IRT_RADIANCE_F32 && desc->radiance_format != IRT_RADIANCE_F16) ||
        (desc->moments_format != IRT_MOMENTS_F32 && desc->moments_format != IRT_MOMENTS_F16)) {
        ctx->set_error("unsupported storage format");
        return IRT_E_INVALID;
    }
    uint64_t need = irt_session_bytes(desc);
    // Admission by HBM bytes against the context budget.
    uint64_t cur = ctx->in_use.load();
    for (;;) {
        if (cur + need > ctx->budget) {
            ctx->set_error("session exceeds the HBM budget");
            return IRT_E_ADMISSION;
        }
        if (ctx->in_use.compare_exchange_weak(cur, cur + need)) break;
    }
    DeviceGuard g(ctx->device);
    irt_session* s = new (std::nothrow) irt_session();
    if (!s) {
        ctx->in_use -= need;
        return IRT_E_NOMEM;
    }
    s->ctx = ctx;
    s->desc = *desc;
    s->W = desc->settings.render_width;
    s->H = desc->settings.render_height;
    s->P = (size_t)s->W * s->H;
    s->rad_bytes = desc->radiance_format == IRT_RADIANCE_F16 ? 8 : 16;
    s->mom_bytes = desc->moments_format == IRT_MOMENTS_F16 ? 8 : 16;
    s->normal_bytes = normal_bytes_of(desc->gbuffer_format);
    s->bytes = need;
    uint64_t used = 0;
    auto fail = [&](irt_status st) {
        irt_session_destroy(s);
        return st;
    };
    const size_t P = s->P;
    for (int k = needs_candidates(*desc) ? 0 : 1; k < 3; k++) {
        irt_status st = dev_alloc(ctx, &s->dres[k], P * 32, used);
        if (st) return fail(st);
        st = dev_alloc(ctx, &s->ires[k], P * 32, used);
        if (st) return fail(st);
    }
    irt_status st = dev_alloc(ctx, &s->archive,
                              (size_t)(desc->settings.restir_max_history + 1) * desc->settings.vpl_count * 48, used);
    if (!st) st = dev_alloc(ctx, &s->prev_depth, P * 4, used);
    if (!st) st = dev_alloc(ctx, &s->prev_normal, P * s->normal_bytes, used);
    if (!st) st = dev_alloc(ctx, &s->direct, P * 16, used);
    if (!st) st = dev_alloc(ctx, &s->noisy, P * s->rad_bytes, used);
    for (int k = 0; k < 2 && !st; k++) {
        st = dev_alloc(ctx, &s->moments[k], P * s->mom_bytes, used);
        if (!st) st = dev_alloc(ctx, &s->feedback[k], P * s->rad_bytes, used);
        if (!st) st = dev_alloc(ctx, &s->scratch[k], P * s->rad_bytes, used);
    }
    if (!st) st = dev_alloc(ctx, &s->temporal, P * s->rad_bytes, used);
    if (!st) st = dev_alloc(ctx, &s->filtered, P * s->rad_bytes, used);
    if (!st) st = dev_alloc(ctx, &s->error, 16, used);
    if (desc->fused == 1) {
        if (!st) st = dev_alloc(ctx, &s->rays, P * 2 * sizeof(RayRecord), used);
        if (!st) st = dev_alloc(ctx, &s->ray_counters, 16, used);
        if (!st) st = dev_alloc(ctx, &s->vis, P * 2 * 4, used);
        if (!st) st = dev_alloc(ctx, &s->pending, P * 2 * 16, used);
    }
    for (int k = 0; k < 2; k++) {
        if (!st) st = dev_alloc(ctx, &s->guide[k], P * 16, used);
    }
    if (!st) st = dev_alloc(ctx, &s->feat, P * 32, used);
    if (!st && cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess)
        st = IRT_E_CUDA;
    if (st) return fail(st);
    *out = s;
    return IRT_OK;
}

static irt_status flush_output(irt_session* s, bool after_march);

void irt_session_destroy(irt_session* s) {
    if (!s) return;
    DeviceGuard g(s->ctx->device);
    // The last call's image still goes to its host buffer, as it would at
    // irt_session_host_sync.
    if (s->pipe.ready) flush_output(s, false);
    void* ptrs[] = {s->dres[0], s->dres[1], s->dres[2], s->ires[0], s->ires[1], s->ires[2], s->archive,
                    s->prev_depth, s->prev_normal, s->direct, s->noisy, s->moments[0], s->moments[1],
                    s->feedback[0], s->feedback[1], s->temporal, s->scratch[0], s->scratch[1], s->filtered, s->error,
                    s->rays, s->ray_counters, s->vis, s->pending, s->guide[0], s->guide[1], s->feat};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->pipe.ready) {
        irt_session::HostPipe& hp = s->pipe;
        if (hp.copy) cudaStreamSynchronize(hp.copy);
        if (hp.copy_out) cudaStreamSynchronize(hp.copy_out);
        for (void* p : {hp.gbuf[0], hp.gbuf[1], (void*)hp.vpls, hp.out[0], hp.out[1]})
            if (p) cudaFree(p);
        for (cudaEvent_t e : {hp.copied[0], hp.copied[1], hp.rendered[0], hp.rendered[1], hp.vpl_free[0],
                              hp.vpl_free[1], hp.vpl_free[2], hp.out_ready[0], hp.out_ready[1], hp.out_done[0],
                              hp.out_done[1], hp.march_done})
            if (e) cudaEventDestroy(e);
        if (hp.copy) cudaStreamDestroy(hp.copy);
        if (hp.copy_out) cudaStreamDestroy(hp.copy_out);
        if (s->ctx->in_use >= hp.bytes) s->ctx->in_use -= hp.bytes;
    }
    if (s->ev_ready)
        for (auto& row : s->ev)
            for (cudaEvent_t e : row) cudaEventDestroy(e);
    if (s->ctx->in_use >= s->bytes) s->ctx->in_use -= s->bytes;
    delete s;
}

static irt_status check_frame(irt_session* s, const irt_frame* f, const irt_gbuffer* g) {
    irt_context* ctx = s->ctx;
    if (!f || !g) return IRT_E_INVALID;
    if (f->size[0] != s->W || f->size[1] != s->H) {
        ctx->set_error("frame size differs from the session's");
        return IRT_E_INVALID;
    }
    if (g->format != s->desc.gbuffer_format || !g->depth || !g->normal || !g->color || !g->params || !g->motion) {
        ctx->set_error("G-buffer format or planes invalid");
        return IRT_E_INVALID;
    }
    return IRT_OK;
}

// Per-pixel world positions of this frame (current depth, inv_vp) and of the
// previous frame's pixels (previous depth, previous_inv_vp).
static cudaError_t compute_guides(irt_session* s, const irt_frame* f, const irt_gbuffer* g, cudaStream_t st) {
    SvgfLaunch G{};
    G.frame = f;
    G.gbuffer = *g;
    G.old_depth = s->prev_depth;
    G.old_normal = s->prev_normal;
    G.out = s->guide[0];
    G.out2 = s->feat;
    G.radiance_f16 = s->desc.radiance_format == IRT_RADIANCE_F16;
    // positions, and for decoded G-buffer formats the edge-stopping features
    cudaError_t e = irt_launch_svgf(G, s->desc.gbuffer_format == IRT_GBUFFER_F32 ? 3 : 6, st);
    if (e != cudaSuccess) return e;
    G.out = s->guide[1];
    e = irt_launch_svgf(G, 4, st);
    if (e == cudaSuccess) s->guide_frame = f->size[2];
    return e;
}

static void mark(irt_session* s, int k, cudaStream_t st) {
    if (s->profiling && s->ev_ready) cudaEventRecord(s->ev[s->prof_slot][k], st);
}

irt_status irt_frame_lighting(irt_session* s, const irt_scene* sc, const irt_frame* f, const irt_gbuffer* g,
                              const irt_vpl* cur, const irt_vpl* prev, void* stream) {
    if (!s || !sc) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    irt_status chk = check_frame(s, f, g);
    if (chk) return chk;
    const irt_settings& set = s->desc.settings;
    if (f->counts[1] != set.vpl_count || f->counts[3] != sc->object_count || f->counts[0] > sc->light_count) {
        ctx->set_error("frame counts differ from the session/scene");
        return IRT_E_INVALID;
    }
    // Loop bounds the kernels take from the frame stay within the ranges
    // Settings::validate admits (src/settings.rs:63-94).
    if (f->restir[0] == 0 || f->restir[0] > 256 || f->restir[1] == 0 || f->restir[1] > 256 || f->restir[2] > 32 ||
        f->restir[3] > 256 || !(f->sdf[0] >= 1.f && f->sdf[0] <= 1024.f) || !(f->sdf[1] > 0.f)) {
        ctx->set_error("frame ReSTIR/SDF parameters out of range");
        return IRT_E_INVALID;
    }
    if (!cur || !prev) {
        ctx->set_error("VPL pools required");
        return IRT_E_INVALID;
    }
    if ((uint32_t)f->rr[2] != set.restir_max_history) {
        ctx->set_error("frame rr.z differs from restir_max_history");
        return IRT_E_INVALID;
    }
    DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    s->prof_slot = (int)(f->size[2] % irt_session::kProfRing);
    s->prof_frame[s->prof_slot] = f->size[2];
    mark(s, 0, st);
    CK(compute_guides(s, f, g, st), "position guides");
    // VPL archive ring slot frame % (H+1) (src/renderer.rs:1873-1884).
    size_t pool = (size_t)set.vpl_count * sizeof(irt_vpl);
    uint32_t slot = f->size[2] % (set.restir_max_history + 1u);
    CK(cudaMemcpyAsync((char*)s->archive + slot * pool, cur, pool, cudaMemcpyDeviceToDevice, st), "archive copy");
    mark(s, 1, st);
    LightingLaunch L{};
    L.frame = f;
    L.gbuffer = *g;
    L.objects = sc->objects;
    L.meshes = sc->meshes;
    L.nodes = sc->nodes;
    L.lights = sc->lights_prep;
    L.atlas = sc->atlas;
    L.sdf_f16 = sc->sdf_f16;
    L.sdf_cells = sc->sdf_cells;
    L.field_filter = scene_field_filter(sc);
    L.error = s->error;
    L.cur_vpls = cur;
    L.prev_vpls = prev;
    L.archive = s->archive;
    L.prev_depth = s->prev_depth;
    L.prev_normal = s->prev_normal;
    for (int k = 0; k < 3; k++) {
        L.dres[k] = s->dres[k];
        L.ires[k] = s->ires[k];
    }
    L.direct_out = s->direct;
    L.noisy_out = s->noisy;
    L.radiance_f16 = s->desc.radiance_format == IRT_RADIANCE_F16;
    L.keep_candidates = s->desc.keep_candidates;
    L.rays = s->rays;
    L.ray_counters = s->ray_counters;
    L.vis = s->vis;
    L.pending = s->pending;
    L.guide = s->guide[0];
    L.old_guide = s->guide[1];
    L.feat = s->desc.gbuffer_format == IRT_GBUFFER_F32 ? nullptr : s->feat;
    if (s->desc.fused == 1) {
        // candidates+temporal -> spatial + resolve set-up (ray queue) ->
        // persistent march -> resolve outputs.
        CK(cudaMemsetAsync(s->ray_counters, 0, 16, st), "ray counters");
        CK(irt_launch_lighting(L, kStageReuse, st), "reuse kernel");
        mark(s, 2, st);
        CK(irt_launch_lighting(L, kStageSpatial, st), "spatial kernel");
        mark(s, 3, st);
        MarchLaunch M{};
        M.frame = f;
        M.objects = sc->objects;
        M.meshes = sc->meshes;
        M.nodes = sc->nodes;
        M.atlas = sc->atlas;
        M.sdf_f16 = sc->sdf_f16;
        M.sdf_cells = sc->sdf_cells;
        M.field_filter = scene_field_filter(sc);
        M.error = s->error;
        M.march_scene = sc->march_scene;
        M.cells = sc->cells;
        for (int a = 0; a < 3; a++) {
            M.grid_org[a] = sc->grid_org[a];
            M.grid_inv[a] = sc->grid_inv[a];
        }
        M.rays = s->rays;
        M.ray_counters = s->ray_counters;
        M.vis = s->vis;
        M.num_sms = s->num_sms;
        M.fast = s->desc.exact_march ? 0 : 1;
        CK(irt_launch_march(M, st), "march kernel");
        if (s->pipe.ready) CK(cudaEventRecord(s->pipe.march_done, st), "pipeline event");
        mark(s, 4, st);
        CK(irt_launch_lighting(L, kStageCombine, st), "combine kernel");
        mark(s, 5, st);
    } else if (s->desc.fused == 2) {
        CK(irt_launch_lighting(L, kStageReuse, st), "reuse kernel");
        mark(s, 2, st);
        CK(irt_launch_lighting(L, kStageShade, st), "shade kernel");
        mark(s, 3, st);
        mark(s, 4, st);
        mark(s, 5, st);
    } else {
        for (int p = 0; p < 4; p++) CK(irt_launch_lighting(L, p, st), "lighting pass");
        mark(s, 2, st);
        for (int p = 4; p < 6; p++) CK(irt_launch_lighting(L, p, st), "lighting pass");
        mark(s, 3, st);
        for (int p = 6; p < 8; p++) CK(irt_launch_lighting(L, p, st), "lighting pass");
        mark(s, 4, st);
        mark(s, 5, st);
    }
    s->last_frame = f->size[2];
    s->have_frame = true;
    return IRT_OK;
}

irt_status irt_frame_svgf(irt_session* s, const irt_frame* f, const irt_gbuffer* g, void* stream) {
    if (!s) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    irt_status chk = check_frame(s, f, g);
    if (chk) return chk;
    DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int cur = (int)(f->size[2] % 2u), old = 1 - cur;
    const size_t rb = s->P * s->rad_bytes;
    if (f->flags[2] >= 3u) {  // debug views bypass SVGF (src/svgf.rs:154-161)
        CK(cudaMemcpyAsync(s->filtered, s->noisy, rb, cudaMemcpyDeviceToDevice, st), "svgf bypass");
        mark(s, 6, st);
        mark(s, 7, st);
        mark(s, 8, st);
    } else {
        // Positions for this frame (already there when the lighting ran).
        if (s->guide_frame != f->size[2]) CK(compute_guides(s, f, g, st), "position guides");
        SvgfLaunch L{};
        L.frame = f;
        L.gbuffer = *g;
        L.old_depth = s->prev_depth;
        L.old_normal = s->prev_normal;
        L.guide = s->guide[0];
        L.old_guide = s->guide[1];
        L.feat = s->feat;
        L.radiance_f16 = s->desc.radiance_format == IRT_RADIANCE_F16;
        L.moments_f16 = s->desc.moments_format == IRT_MOMENTS_F16;
        L.in = s->noisy;
        L.aux = s->feedback[old];
        L.moments_in = s->moments[old];
        L.out = s->temporal;
        L.moments_out = s->moments[cur];
        CK(irt_launch_svgf(L, 0, st), "svgf temporal");
        mark(s, 6, st);
        L.in = s->temporal;
        L.moments_in = s->moments[cur];
        L.out = s->scratch[0];
        CK(irt_launch_svgf(L, 1, st), "svgf variance");
        mark(s, 7, st);
        // A-trous ping-pong: iteration 0 writes feedback[cur] directly (the
        // reference copies scratch[1] there), the last writes the output.
        const uint32_t iters = s->desc.settings.svgf_iterations;
        const void* in = s->scratch[0];
        for (uint32_t i = 0; i < iters; i++) {
            void* out;
            void* out2 = nullptr;
            if (i + 1 == iters) {
                out = s->filtered;
                if (i == 0) out2 = s->feedback[cur];
            } else {
                out = i == 0 ? s->feedback[cur] : s->scratch[i % 2];
            }
            L.in = in;
            L.out = out;
            L.out2 = out2;
            L.step = 1 << i;
            CK(irt_launch_svgf(L, 2, st), "svgf atrous");
            in = out;
        }
        mark(s, 8, st);
    }
    // Depth/normal history for the next frame (src/renderer.rs:1951-1960).
    CK(cudaMemcpyAsync(s->prev_depth, g->depth, s->P * 4, cudaMemcpyDeviceToDevice, st), "depth history");
    CK(cudaMemcpyAsync(s->prev_normal, g->normal, s->P * s->normal_bytes, cudaMemcpyDeviceToDevice, st),
       "normal history");
    mark(s, 9, st);
    return IRT_OK;
}

irt_status irt_render_frame(irt_session* s, const irt_scene* sc, const irt_frame* f, const irt_gbuffer* g,
                            const irt_vpl* cur, const irt_vpl* prev, void* stream) {
    irt_status r = irt_frame_lighting(s, sc, f, g, cur, prev, stream);
    if (r) return r;
    return irt_frame_svgf(s, f, g, stream);
}

// ------------------------------------------------------------------ host inputs
static uint64_t plane_bytes(int fmt, int k, size_t P) {
    static const uint64_t b[3][5] = {{4, 16, 16, 8, 8}, {4, 8, 8, 4, 4}, {4, 4, 4, 4, 4}};
    return b[fmt][k] * P;
}

static irt_status pipe_setup(irt_session* s) {
    irt_context* ctx = s->ctx;
    irt_session::HostPipe& hp = s->pipe;
    const size_t P = s->P;
    const int fmt = s->desc.gbuffer_format;
    uint64_t gb = 0;
    for (int k = 0; k < 5; k++) gb += plane_bytes(fmt, k, P);
    const uint64_t pool = (uint64_t)s->desc.settings.vpl_count * sizeof(irt_vpl);
    const uint64_t need = 2 * gb + 4 * pool + 2 * P * s->rad_bytes;
    uint64_t cur = ctx->in_use.load();
    for (;;) {
        if (cur + need > ctx->budget) {
            ctx->set_error("host-input staging exceeds the HBM budget");
            return IRT_E_ADMISSION;
        }
        if (ctx->in_use.compare_exchange_weak(cur, cur + need)) break;
    }
    hp.bytes = need;
    hp.ready = true;  // from here irt_session_destroy releases what exists
    uint64_t used = 0;
    CK(cudaStreamCreateWithFlags(&hp.copy, cudaStreamNonBlocking), "copy stream");
    CK(cudaStreamCreateWithFlags(&hp.copy_out, cudaStreamNonBlocking), "copy stream");
    for (int k = 0; k < 2; k++) {
        irt_status st = dev_alloc(ctx, &hp.gbuf[k], gb, used);
        if (!st) st = dev_alloc(ctx, &hp.out[k], P * s->rad_bytes, used);
        if (st) return st;
    }
    irt_status st = dev_alloc(ctx, &hp.vpls, 4 * pool, used);  // zero-filled: pool [3] stays zero
    if (st) return st;
    for (cudaEvent_t* e : {&hp.copied[0], &hp.copied[1], &hp.rendered[0], &hp.rendered[1], &hp.vpl_free[0],
                           &hp.vpl_free[1], &hp.vpl_free[2], &hp.out_ready[0], &hp.out_ready[1], &hp.out_done[0],
                           &hp.out_done[1], &hp.march_done})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "pipeline events");
    return IRT_OK;
}

// Queues the host copy of the last call's image (after the latest march
// when `after_march`).
static irt_status flush_output(irt_session* s, bool after_march) {
    irt_context* ctx = s->ctx;
    irt_session::HostPipe& hp = s->pipe;
    if (!hp.pending_out) return IRT_OK;
    const int slot = hp.pending_slot;
    CK(cudaStreamWaitEvent(hp.copy_out, hp.out_ready[slot], 0), "pipeline wait");
    if (after_march) CK(cudaStreamWaitEvent(hp.copy_out, hp.march_done, 0), "pipeline wait");
    CK(cudaMemcpyAsync(hp.pending_out, hp.out[slot], s->P * s->rad_bytes, cudaMemcpyDeviceToHost, hp.copy_out),
       "output");
    CK(cudaEventRecord(hp.out_done[slot], hp.copy_out), "pipeline event");
    hp.pending_out = nullptr;
    return IRT_OK;
}

irt_status irt_render_frame_host(irt_session* s, const irt_scene* sc, const irt_frame* f, const irt_gbuffer* host_g,
                                 const irt_vpl* host_vpls, void* out_host, void* stream) {
    if (!s || !sc || !f || !host_g || !host_vpls) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    if (host_g->format != s->desc.gbuffer_format || !host_g->depth || !host_g->normal || !host_g->color ||
        !host_g->params || !host_g->motion) {
        ctx->set_error("G-buffer format or planes invalid");
        return IRT_E_INVALID;
    }
    DeviceGuard dg(ctx->device);
    irt_session::HostPipe& hp = s->pipe;
    if (!hp.ready) {
        irt_status st = pipe_setup(s);
        if (st) return st;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t P = s->P;
    const int fmt = s->desc.gbuffer_format;
    const int slot = (int)(hp.calls % 2u);
    const int vslot = (hp.last_vpl + 1) % 3;
    // Inputs, on the copy stream: the G-buffer slot and the VPL pool may be
    // overwritten once the frames that read them have rendered.
    CK(cudaStreamWaitEvent(hp.copy, hp.rendered[slot], 0), "pipeline wait");
    CK(cudaStreamWaitEvent(hp.copy, hp.vpl_free[vslot], 0), "pipeline wait");
    // Uploads run after the previous frame's march, beside its SVGF passes:
    // the copies stream through L2, and during the march (which lives on
    // L2-resident scene records, leaf cache and SDF texels) they slowed the
    // frame by more than the copy takes.
    CK(cudaStreamWaitEvent(hp.copy, hp.march_done, 0), "pipeline wait");
    const void* src[5] = {host_g->depth, host_g->normal, host_g->color, host_g->params, host_g->motion};
    char* base = static_cast<char*>(hp.gbuf[slot]);
    const void* dst[5];
    uint64_t off = 0;
    for (int k = 0; k < 5; k++) {
        dst[k] = base + off;
        CK(cudaMemcpyAsync(base + off, src[k], plane_bytes(fmt, k, P), cudaMemcpyHostToDevice, hp.copy), "G-buffer in");
        off += plane_bytes(fmt, k, P);
    }
    const uint64_t pool = (uint64_t)s->desc.settings.vpl_count * sizeof(irt_vpl);
    irt_vpl* cur = hp.vpls + (size_t)vslot * s->desc.settings.vpl_count;
    const irt_vpl* prev = hp.last_vpl < 0 ? hp.vpls + 3ull * s->desc.settings.vpl_count
                                          : hp.vpls + (size_t)hp.last_vpl * s->desc.settings.vpl_count;
    CK(cudaMemcpyAsync(cur, host_vpls, pool, cudaMemcpyHostToDevice, hp.copy), "VPLs in");
    CK(cudaEventRecord(hp.copied[slot], hp.copy), "pipeline event");
    // The frame, on the caller's stream, once its inputs have landed.
    CK(cudaStreamWaitEvent(st, hp.copied[slot], 0), "pipeline wait");
    irt_gbuffer g{fmt, static_cast<const float*>(dst[0]), dst[1], dst[2], dst[3], dst[4]};
    irt_status r = irt_render_frame(s, sc, f, &g, cur, prev, stream);
    if (r) return r;
    CK(cudaEventRecord(hp.rendered[slot], st), "pipeline event");
    // The pool this frame read as `previous` is free after it; the current
    // one is the next frame's previous.
    if (hp.last_vpl >= 0) CK(cudaEventRecord(hp.vpl_free[hp.last_vpl], st), "pipeline event");
    // The previous call's image goes to the host after this frame's march,
    // beside this frame's SVGF passes (and the next inputs), like the uploads:
    // during the march the copy's traffic through L2 slows it.
    irt_status fr = flush_output(s, true);
    if (fr) return fr;
    if (out_host) {
        // A device copy of the output (the next frame overwrites the image);
        // its host copy is queued by the next call or irt_session_host_sync.
        CK(cudaStreamWaitEvent(st, hp.out_done[slot], 0), "pipeline wait");
        CK(cudaMemcpyAsync(hp.out[slot], s->filtered, P * s->rad_bytes, cudaMemcpyDeviceToDevice, st), "output");
        CK(cudaEventRecord(hp.out_ready[slot], st), "pipeline event");
        hp.pending_out = out_host;
        hp.pending_slot = slot;
    }
    hp.last_vpl = vslot;
    hp.calls++;
    return IRT_OK;
}

irt_status irt_session_host_sync(irt_session* s, void* stream) {
    if (!s) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    if (!s->pipe.ready) return IRT_OK;
    DeviceGuard dg(ctx->device);
    irt_status fr = flush_output(s, false);
    if (fr) return fr;
    if (!stream) {
        CK(cudaStreamSynchronize(s->pipe.copy), "host inputs");
        CK(cudaStreamSynchronize(s->pipe.copy_out), "host outputs");
        return IRT_OK;
    }
    for (cudaStream_t c : {s->pipe.copy, s->pipe.copy_out}) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "host join");
        cudaError_t r = cudaEventRecord(e, c);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), e, 0);
        cudaEventDestroy(e);
        CK(r, "host join");
    }
    return IRT_OK;
}

irt_status irt_session_buffer(irt_session* s, int32_t which, void** ptr, uint64_t* bytes) {
    if (!s || !ptr || !bytes) return IRT_E_INVALID;
    const size_t P = s->P;
    const int cur = (int)(s->last_frame % 2u), old = 1 - cur;
    void* p = nullptr;
    uint64_t b = 0;
    switch (which) {
    case IRT_BUF_DIRECT: p = s->direct; b = P * 16; break;
    case IRT_BUF_NOISY: p = s->noisy; b = P * s->rad_bytes; break;
    case IRT_BUF_FILTERED: p = s->filtered; b = P * s->rad_bytes; break;
    case IRT_BUF_MOMENTS: p = s->moments[cur]; b = P * s->mom_bytes; break;
    case IRT_BUF_MOMENTS_OLD: p = s->moments[old]; b = P * s->mom_bytes; break;
    case IRT_BUF_FEEDBACK: p = s->feedback[cur]; b = P * s->rad_bytes; break;
    case IRT_BUF_FEEDBACK_OLD: p = s->feedback[old]; b = P * s->rad_bytes; break;
    case IRT_BUF_VPL_ARCHIVE:
        p = s->archive;
        b = (uint64_t)(s->desc.settings.restir_max_history + 1) * s->desc.settings.vpl_count * 48;
        break;
    case IRT_BUF_PREV_DEPTH: p = s->prev_depth; b = P * 4; break;
    case IRT_BUF_PREV_NORMAL: p = s->prev_normal; b = P * s->normal_bytes; break;
    case IRT_BUF_ERROR: p = s->error; b = 16; break;
    case IRT_BUF_TEMPORAL: p = s->temporal; b = P * s->rad_bytes; break;
    case IRT_BUF_VARIANCE: p = s->scratch[0]; b = P * s->rad_bytes; break;
    default: break;
    }
    if (which == IRT_BUF_RES_DIRECT || which == IRT_BUF_RES_INDIRECT) {
        // Three separate allocations: report [2] (the final reservoirs); [0]
        // and [1] are reachable through irt_session_reservoirs.
        irt_reservoir** set = which == IRT_BUF_RES_DIRECT ? s->dres : s->ires;
        p = set[2];
        b = P * 32;
    }
    if (!p) return IRT_E_INVALID;
    *ptr = p;
    *bytes = b;
    return IRT_OK;
}

irt_status irt_session_check(irt_session* s, void* stream) {
    if (!s) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    DeviceGuard dg(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t h[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(h, s->error, 16, cudaMemcpyDeviceToHost, st), "error word");
    CK(cudaStreamSynchronize(st), "sync");
    CK(cudaMemsetAsync(s->error, 0, 16, st), "error clear");
    if (h[0]) {
        char buf[96];
        std::snprintf(buf, sizeof(buf), "device error word 0x%x", h[0]);
        ctx->set_error(buf);
        return IRT_E_DEVICE;
    }
    return IRT_OK;
}

irt_status irt_session_set_profiling(irt_session* s, int32_t on) {
    if (!s) return IRT_E_INVALID;
    irt_context* ctx = s->ctx;
    if (on && !s->ev_ready) {
        DeviceGuard dg(ctx->device);
        for (auto& row : s->ev)
            for (cudaEvent_t& e : row) CK(cudaEventCreate(&e), "event");
        s->ev_ready = true;
    }
    s->profiling = on != 0;
    return IRT_OK;
}

// Device time of one profiled frame's stages (ms): archive copy, candidates +
// temporal, spatial + resolve, SVGF temporal, SVGF variance, a-trous,
// history copy, total.  Synchronises on that frame's last event.  Frames
// older than the ring (128 frames) are overwritten.
irt_status irt_session_pass_ms_at(irt_session* s, uint32_t frame_index, float out_ms[10]) {
    if (!s || !out_ms || !s->ev_ready) return IRT_E_STATE;
    irt_context* ctx = s->ctx;
    int slot = (int)(frame_index % irt_session::kProfRing);
    if (s->prof_frame[slot] != frame_index) {
        ctx->set_error("frame not in the profiling ring");
        return IRT_E_STATE;
    }
    DeviceGuard dg(ctx->device);
    cudaEvent_t* e = s->ev[slot];
    const int last = irt_session::kProfEvents - 1;
    CK(cudaEventSynchronize(e[last]), "event sync");
    for (int k = 0; k < last; k++) CK(cudaEventElapsedTime(&out_ms[k], e[k], e[k + 1]), "elapsed");
    CK(cudaEventElapsedTime(&out_ms[last], e[0], e[last]), "elapsed");
    return IRT_OK;
}

irt_status irt_session_pass_ms(irt_session* s, float out_ms[10]) {
    if (!s) return IRT_E_INVALID;
    return irt_session_pass_ms_at(s, s->last_frame, out_ms);
}

// Reservoir set k (0, 1, 2) of a domain (0 direct, 1 indirect).
irt_status irt_session_reservoirs(irt_session* s, int32_t domain, int32_t k, void** ptr, uint64_t* bytes) {
    if (!s || !ptr || !bytes || domain < 0 || domain > 1 || k < 0 || k > 2) return IRT_E_INVALID;
    irt_reservoir* p = domain == 0 ? s->dres[k] : s->ires[k];
    if (!p) return IRT_E_STATE;
    *ptr = p;
    *bytes = s->P * 32;
    return IRT_OK;
}


}  // extern "C"
