// kernels.h — host-side launch descriptors of the lighting and SVGF kernels.
#pragma once
#include <cuda_runtime.h>

#include "../../include/irt.h"

// Lighting stages: 0..7 are the reference entry points in schedule order
// (candidates_direct, candidates_indirect, temporal_direct, temporal_indirect,
// spatial_direct, spatial_indirect, resolve_direct, resolve_indirect).
constexpr int kStageReuse = 100;  // fused 0..3
constexpr int kStageShade = 101;  // fused 4..7

struct LightingLaunch {
    const irt_frame* frame;
    irt_gbuffer gbuffer;
    const irt_object* objects;
    const irt_mesh* meshes;
    const irt_node* nodes;
    const irt_light* lights;
    cudaTextureObject_t atlas;
    int sdf_f16;
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
};

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
};

cudaError_t irt_launch_lighting(const LightingLaunch& L, int stage, cudaStream_t st);
cudaError_t irt_launch_svgf(const SvgfLaunch& L, int stage, cudaStream_t st);
