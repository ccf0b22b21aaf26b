// capi_internal.h — the library's context, scene and session objects and
// the helpers the C-ABI translation units share (capi.cu, batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "dev_sdf.cuh"
#include "kernels.h"

struct irt_context {
    int device = 0;
    uint64_t budget = 0;
    std::atomic<uint64_t> in_use{0};
    mutable std::mutex mu;
    std::string last_error;
    void set_error(const std::string& e) {
        std::lock_guard<std::mutex> g(mu);
        last_error = e;
    }
};

struct irt_scene {
    irt_context* ctx = nullptr;
    uint32_t mesh_count = 0;
    irt_mesh* meshes = nullptr;
    cudaArray_t atlas_array = nullptr;
    cudaTextureObject_t atlas = 0;
    // The same atlas through a linear sampler at normalised coordinates, for
    // the reference's filtered sample_field (IRT_FIELD_LINEAR).
    cudaTextureObject_t atlas_linear = 0;
    int field_linear = 0;            // in use since the last irt_scene_update
    int field_linear_requested = 0;  // irt_scene_set_field_filter, applied by the next update
    int sdf_f16 = 0;
    uint32_t atlas_dims[3] = {0, 0, 0};
    // Corner cells: per field mesh, the 8 corner texels of each of its
    // (res-1)^3 cells in one record (f32: 32 B, f16: 16 B); a mesh's first
    // cell index is in hi[3] of its rows (host_meshes and the device copy).
    void* sdf_cells = nullptr;
    std::vector<irt_mesh> host_meshes;
    // per-frame data
    irt_object* objects = nullptr;
    irt_node* nodes = nullptr;
    irt_light* lights = nullptr;
    irt_light* lights_prep = nullptr;  // spot direction normalised, cos(angle / 2)
    uint32_t object_cap = 0, light_cap = 0;
    // compact march scene (nodes + object records with their mesh folded in)
    float4* march_scene = nullptr;
    std::vector<float4> march_host;
    // Pinned staging of the per-frame uploads, two slots used in turn, so an
    // update neither waits for the device nor races an earlier copy.
    unsigned char* pinned[2] = {nullptr, nullptr};
    size_t pinned_cap[2] = {0, 0};
    cudaEvent_t pinned_free[2] = {nullptr, nullptr};
    uint32_t updates = 0;
    // leaf-order cache (rebuilt when the BVH changes)
    uint4* cells = nullptr;
    float* corners = nullptr;
    size_t corner_cap = 0;
    std::vector<irt_node> cached_nodes;
    std::vector<irt_object> cached_objects;
    float grid_org[3] = {0, 0, 0}, grid_inv[3] = {0, 0, 0};
    uint32_t object_count = 0, light_count = 0;
    uint64_t bytes = 0;
};

// The field sampler the kernels use for a scene (point-sampled trilinear or
// the hardware-linear fetch).
inline irtd::FieldFilter scene_field_filter(const irt_scene* sc) {
    irtd::FieldFilter f{};
    f.linear = sc->field_linear ? sc->atlas_linear : 0;
    for (int a = 0; a < 3; a++) f.dims[a] = (float)sc->atlas_dims[a];
    return f;
}

struct irt_session {
    irt_context* ctx = nullptr;
    irt_session_desc desc{};
    uint32_t W = 0, H = 0;
    size_t P = 0;
    size_t rad_bytes = 0, normal_bytes = 0, mom_bytes = 0;
    irt_reservoir* dres[3] = {nullptr, nullptr, nullptr};
    irt_reservoir* ires[3] = {nullptr, nullptr, nullptr};
    irt_vpl* archive = nullptr;
    float* prev_depth = nullptr;
    void* prev_normal = nullptr;
    float4* direct = nullptr;
    void* noisy = nullptr;
    float4* moments[2] = {nullptr, nullptr};
    void* feedback[2] = {nullptr, nullptr};
    void* temporal = nullptr;
    void* scratch[2] = {nullptr, nullptr};
    void* filtered = nullptr;
    uint32_t* error = nullptr;
    uint64_t bytes = 0;
    uint32_t last_frame = 0;
    bool have_frame = false;
    bool profiling = false;
    // Profiling: a ring of kProfRing frames x 8 stage-boundary events, so a
    // long timed run can be read back afterwards without per-frame syncs.
    static constexpr int kProfRing = 128;
    static constexpr int kProfEvents = 10;
    cudaEvent_t ev[kProfRing][kProfEvents] = {};
    // ray-queue resolve buffers
    RayRecord* rays = nullptr;
    uint32_t* ray_counters = nullptr;
    float* vis = nullptr;
    float4* pending = nullptr;
    // per-pixel world positions: [0] this frame, [1] the previous frame's
    // pixels from the previous depth and previous_inv_vp
    float4* guide[2] = {nullptr, nullptr};
    float4* feat = nullptr;  // this frame's SVGF edge-stopping features, 2 float4 per pixel
    uint32_t guide_frame = 0xffffffffu;
    int num_sms = 0;
    // Host-input pipeline (irt_render_frame_host), created on first use:
    // a copy stream, double-buffered device G-buffers, three VPL pools plus
    // a zero pool, double-buffered device copies of the output image.
    struct HostPipe {
        bool ready = false;
        cudaStream_t copy = nullptr;      // host -> device inputs
        cudaStream_t copy_out = nullptr;  // device -> host outputs (own stream: an output copy
                                          // waits for its frame, the next inputs must not)
        void* gbuf[2] = {nullptr, nullptr};
        irt_vpl* vpls = nullptr;      // 4 pools: [0..2] ring, [3] zeros
        void* out[2] = {nullptr, nullptr};
        cudaEvent_t copied[2] = {}, rendered[2] = {}, vpl_free[3] = {}, out_ready[2] = {}, out_done[2] = {};
        cudaEvent_t march_done = nullptr;  // after the last frame's march (recorded by irt_frame_lighting)
        void* pending_out = nullptr;        // host destination of the last call's image, copied at the next call
        int pending_slot = 0;               // ... from out[pending_slot]
        uint32_t calls = 0;
        int last_vpl = -1;
        uint64_t bytes = 0;
    } pipe;
    bool ev_ready = false;
    int prof_slot = 0;
    uint32_t prof_frame[kProfRing] = {};
};

namespace {

uint32_t normal_bytes_of(int fmt) {
    return fmt == IRT_GBUFFER_F32 ? 16u : (fmt == IRT_GBUFFER_F16 ? 8u : 4u);
}

irt_status cuda_fail(irt_context* ctx, cudaError_t e, const char* what) {
    if (ctx) ctx->set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return IRT_E_CUDA;
}

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

template <class T>
irt_status dev_alloc(irt_context* ctx, T** p, size_t bytes, uint64_t& counter) {
    if (bytes == 0) {
        *p = nullptr;
        return IRT_OK;
    }
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    e = cudaMemset(q, 0, bytes);
    if (e != cudaSuccess) {
        cudaFree(q);
        return cuda_fail(ctx, e, "cudaMemset");
    }
    *p = static_cast<T*>(q);
    counter += bytes;
    return IRT_OK;
}

bool needs_candidates(const irt_session_desc& d) { return d.keep_candidates || !d.fused; }

}  // namespace
