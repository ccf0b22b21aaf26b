// batch.cu — batched views (irt_batch_* in irt.h): one launch per pass over
// every view, per-view argument tables on the device, a CUDA graph per frame
// parity, and an autotuner for the tile shapes.
//
// Per frame the schedule is the single-session schedule 1 of
// irt_frame_lighting + irt_frame_svgf, each step as one batched launch:
//   frame upload (pinned -> device table), position guides (this frame and
//   the previous), VPL archive slot copy + ray-counter reset, reuse, spatial
//   + ray emission, march (views grouped by scene), combine, SVGF temporal,
//   variance, a-trous x iterations, depth/normal history copy.
// The per-view tables hold the same pointers the single-session path passes
// as kernel parameters, so every view's results are identical to rendering
// it alone.  Tables depend on the frame parity (SVGF ping-pong) and on the
// caller's buffers; they are rebuilt (and graphs re-captured) when any
// pointer or scene layout changes.
// Views run in waves: consecutive views whose pixels add up to at most the
// wave budget share one launch per pass, and the waves run one after
// another, so a wave's buffers are still in L2 when its next pass reads them
// (running every view pass by pass streams the whole batch through HBM
// between passes).  The autotuner picks the wave budget (one wave = all
// views) together with the tile shapes.  The batch works on a stream of its own
// (a graph cannot be captured on the legacy default stream) that is joined
// to the caller's stream with events in both directions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "capi_internal.h"

namespace {

struct Shape {
    uint32_t bx, by;
};
const Shape kShapes[] = {{32, 8}, {64, 4}, {16, 16}, {128, 2}, {256, 1}};
constexpr int kNumShapes = 5;
const int kMarchBps[] = {0, 5, 4};  // CTAs per SM for the march (0 = occupancy maximum)
constexpr int kNumMarch = 3;
// Wave budgets in pixels (0 = every view in one wave).
const uint64_t kWavePx[] = {0, 8u << 20, 4u << 20, 2u << 20, 1u << 20};
constexpr int kNumWaves = 5;

// Tuned passes (2-D kernels).
enum { kTReuse = 0, kTSpatial, kTTemporal, kTVariance, kTAtrous, kNumTuned };
const char* const kTunedNames[kNumTuned] = {"reuse", "spatial", "temporal", "variance", "atrous"};
// Pass-time slots of irt_batch_pass_ms.
enum { kPGuides = 0, kPArchive, kPReuse, kPSpatial, kPMarch, kPCombine, kPTemporal, kPVariance, kPAtrous, kPHistory,
       kPTotal, kPGraph, kNumPass };
// Events of a timed frame: before the upload, after each of the 11 steps.
constexpr int kNumEvents = 12;

struct ParityTables {
    bool valid = false;
    std::vector<uintptr_t> signature;
    void* largs = nullptr;         // LightArgs x n
    void* sviews[8] = {};          // SVGF records x n: temporal, variance, a-trous 0..3, guides, previous guides
    void* history = nullptr;       // history-copy records x n
    MarchGroup* groups = nullptr;  // device, grouped by wave
    MarchQueue* queues = nullptr;  // device
    std::vector<uint32_t> wave_groups;  // groups of wave w: [wave_groups[w], wave_groups[w + 1])
    uint32_t max_scene_bytes = 0;
    cudaGraphExec_t graph = nullptr;
    int renders = 0;               // direct renders of this parity since the tables were built
};

}  // namespace

struct irt_batch {
    irt_context* ctx = nullptr;
    irt_batch_desc desc{};
    uint32_t n = 0;
    std::vector<uint32_t> W, H, vpls;
    std::vector<irt_session*> sess;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t join_in = nullptr, join_out = nullptr;
    // frames: pinned staging per parity and the device table
    irt_frame* h_frames[2] = {nullptr, nullptr};
    irt_frame* d_frames = nullptr;
    cudaEvent_t staged[2] = {nullptr, nullptr};  // the last use of h_frames[p] completed
    // tile tables: 2-D per candidate shape, 1-D (256 pixels)
    // per wave w: n_w + 1 block offsets at entry wave_begin[w] + w
    uint32_t* d_tiles2[kNumShapes] = {};
    std::vector<uint32_t> tiles2[kNumShapes];
    uint32_t* d_tiles1 = nullptr;
    std::vector<uint32_t> tiles1;
    std::vector<uint32_t> wave_begin;  // views of wave w: [wave_begin[w], wave_begin[w + 1])
    uint64_t wave_budget = 0;         // pixels per wave (0 = all views in one wave)
    size_t la = 0, sv = 0;             // bytes of a lighting / SVGF per-view record
    ParityTables par[2];
    // tuning
    int shape_of[kNumTuned] = {0, 0, 0, 0, 0};
    int march_choice = 0;
    uint32_t tune_left = 0, tune_total = 0;
    std::vector<double> tune_ms;  // [candidate][kNumTuned + 1]
    std::vector<int> tune_count;
    double wave_ms[kNumWaves] = {};
    int wave_count[kNumWaves] = {};
    int tune_wave = -1;  // wave candidate being timed after the shapes (-1: none)
    cudaEvent_t ev[kNumEvents] = {};
    float pass_ms[kNumPass] = {};
    bool timed_pending = false;
};

namespace {

template <class T>
cudaError_t upload(T** dst, const void* src, size_t bytes) {
    if (!*dst) {
        cudaError_t e = cudaMalloc(dst, bytes);
        if (e != cudaSuccess) return e;
    }
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
}

void free_tables(ParityTables& t) {
    if (t.graph) cudaGraphExecDestroy(t.graph);
    t.graph = nullptr;
    if (t.largs) cudaFree(t.largs);
    for (void*& p : t.sviews) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    if (t.history) cudaFree(t.history);
    if (t.groups) cudaFree(t.groups);
    if (t.queues) cudaFree(t.queues);
    t.largs = t.history = nullptr;
    t.groups = nullptr;
    t.queues = nullptr;
    t.wave_groups.clear();
    t.valid = false;
    t.renders = 0;
}

LightingLaunch lighting_launch(irt_session* s, const irt_scene* sc, const irt_frame* f, const irt_gbuffer& g,
                               const irt_vpl* cur, const irt_vpl* prev) {
    LightingLaunch L{};
    L.frame = f;
    L.gbuffer = g;
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
    L.keep_candidates = 0;
    L.rays = s->rays;
    L.ray_counters = s->ray_counters;
    L.vis = s->vis;
    L.pending = s->pending;
    L.guide = s->guide[0];
    L.old_guide = s->guide[1];
    L.feat = s->desc.gbuffer_format == IRT_GBUFFER_F32 ? nullptr : s->feat;
    return L;
}

SvgfLaunch svgf_base(irt_session* s, const irt_gbuffer& g) {
    SvgfLaunch L{};
    L.gbuffer = g;
    L.old_depth = s->prev_depth;
    L.old_normal = s->prev_normal;
    L.guide = s->guide[0];
    L.old_guide = s->guide[1];
    L.feat = s->feat;
    L.radiance_f16 = s->desc.radiance_format == IRT_RADIANCE_F16;
    L.moments_f16 = s->desc.moments_format == IRT_MOMENTS_F16;
    return L;
}

std::vector<uintptr_t> signature_of(const irt_batch* b, irt_scene* const* scenes, const irt_frame* frames,
                                    const irt_gbuffer* g, const irt_vpl* const* cur, const irt_vpl* const* prev) {
    std::vector<uintptr_t> sig;
    for (uint32_t v = 0; v < b->n; v++) {
        const irt_scene* sc = scenes[v];
        uintptr_t vals[] = {(uintptr_t)sc, (uintptr_t)sc->objects, (uintptr_t)sc->meshes, (uintptr_t)sc->nodes,
                            (uintptr_t)sc->lights_prep, (uintptr_t)sc->atlas, (uintptr_t)sc->march_scene,
                            (uintptr_t)sc->cells, sc->object_count, (uintptr_t)g[v].depth, (uintptr_t)g[v].normal,
                            (uintptr_t)g[v].color, (uintptr_t)g[v].params, (uintptr_t)g[v].motion,
                            (uintptr_t)cur[v], (uintptr_t)prev[v], frames[v].counts[0], frames[v].counts[3]};
        sig.insert(sig.end(), std::begin(vals), std::end(vals));
        uint32_t gi[6];
        std::memcpy(gi, sc->grid_org, 12);
        std::memcpy(gi + 3, sc->grid_inv, 12);
        sig.insert(sig.end(), std::begin(gi), std::end(gi));
    }
    return sig;
}

irt_status build_tables(irt_batch* b, int p, irt_scene* const* scenes, const irt_frame* frames,
                        const irt_gbuffer* g, const irt_vpl* const* cur, const irt_vpl* const* prev) {
    irt_context* ctx = b->ctx;
    ParityTables& t = b->par[p];
    free_tables(t);
    const int cur_i = p, old_i = 1 - p;
    const size_t la = b->la, sv = b->sv;
    std::vector<unsigned char> hl(la * b->n);
    std::vector<std::vector<unsigned char>> hs(9, std::vector<unsigned char>(sv * b->n));
    const uint32_t iters = b->desc.settings.svgf_iterations;
    for (uint32_t v = 0; v < b->n; v++) {
        irt_session* s = b->sess[v];
        LightingLaunch L = lighting_launch(s, scenes[v], &frames[v], g[v], cur[v], prev[v]);
        irt_lighting_args_fill(L, hl.data() + la * v);
        const SvgfLaunch S = svgf_base(s, g[v]);
        SvgfLaunch T = S;  // temporal
        T.in = s->noisy;
        T.aux = s->feedback[old_i];
        T.moments_in = s->moments[old_i];
        T.out = s->temporal;
        T.moments_out = s->moments[cur_i];
        irt_svgf_view_fill(T, hs[0].data() + sv * v);
        SvgfLaunch V = S;  // variance
        V.in = s->temporal;
        V.moments_in = s->moments[cur_i];
        V.out = s->scratch[0];
        irt_svgf_view_fill(V, hs[1].data() + sv * v);
        // a-trous iterations: the ping-pong of irt_frame_svgf
        const void* in = s->scratch[0];
        for (uint32_t i = 0; i < 4; i++) {
            SvgfLaunch A = S;
            if (i < iters) {
                void* out;
                void* out2 = nullptr;
                if (i + 1 == iters) {
                    out = s->filtered;
                    if (i == 0) out2 = s->feedback[cur_i];
                } else {
                    out = i == 0 ? s->feedback[cur_i] : s->scratch[i % 2];
                }
                A.in = in;
                A.out = out;
                A.out2 = out2;
                A.step = 1 << i;
                in = out;
            }
            irt_svgf_view_fill(A, hs[2 + i].data() + sv * v);
        }
        SvgfLaunch G0 = S;  // positions and edge-stopping features of this frame
        G0.in = g[v].depth;
        G0.out = s->guide[0];
        G0.out2 = s->feat;
        irt_svgf_view_fill(G0, hs[6].data() + sv * v);
        SvgfLaunch G1 = S;  // positions of the previous frame's pixels
        G1.in = s->prev_depth;
        G1.out = s->guide[1];
        irt_svgf_view_fill(G1, hs[7].data() + sv * v);
        SvgfLaunch Hh = S;  // depth / normal history
        Hh.in = g[v].depth;
        Hh.aux = g[v].normal;
        Hh.out = s->prev_depth;
        Hh.out2 = s->prev_normal;
        irt_svgf_view_fill(Hh, hs[8].data() + sv * v);
    }
    CK(upload(&t.largs, hl.data(), hl.size()), "batch lighting table");
    for (int k = 0; k < 8; k++) CK(upload(&t.sviews[k], hs[k].data(), hs[k].size()), "batch svgf table");
    CK(upload(&t.history, hs[8].data(), hs[8].size()), "batch history table");
    // March: per wave, its views grouped by scene (groups in order of first
    // appearance); a group's queues are its views' ray queues.
    std::vector<MarchGroup> groups;
    std::vector<MarchQueue> queues;
    t.max_scene_bytes = 0;
    t.wave_groups.assign(1, 0);
    for (size_t w = 0; w + 1 < b->wave_begin.size(); w++) {
        const uint32_t v0 = b->wave_begin[w], v1 = b->wave_begin[w + 1];
        std::vector<const irt_scene*> order;
        for (uint32_t v = v0; v < v1; v++)
            if (std::find(order.begin(), order.end(), scenes[v]) == order.end()) order.push_back(scenes[v]);
        for (const irt_scene* sc : order) {
            MarchGroup G{};
            G.q_begin = (uint32_t)queues.size();
            for (uint32_t v = v0; v < v1; v++) {
                if (scenes[v] != sc) continue;
                if (queues.size() == G.q_begin) G.f = frames[v];
                irt_session* s = b->sess[v];
                queues.push_back(MarchQueue{s->rays, s->ray_counters, s->vis, (uint32_t)(2 * s->P)});
                if (!G.error) G.error = s->error;
            }
            G.q_end = (uint32_t)queues.size();
            G.objects = sc->objects;
            G.meshes = sc->meshes;
            G.nodes = sc->nodes;
            G.atlas = sc->atlas;
            G.sdf_f16 = sc->sdf_f16;
            G.sdf_cells = sc->sdf_cells;
            G.field_filter = scene_field_filter(sc);
            G.march_scene = sc->march_scene;
            const uint32_t bytes = irt_march_scene_bytes(sc->object_count);
            G.scene_vec4 = bytes / 16;
            t.max_scene_bytes = std::max(t.max_scene_bytes, bytes);
            G.cells = sc->cells;
            for (int a = 0; a < 3; a++) {
                G.grid_org[a] = sc->grid_org[a];
                G.grid_inv[a] = sc->grid_inv[a];
            }
            groups.push_back(G);
        }
        t.wave_groups.push_back((uint32_t)groups.size());
    }
    CK(upload(&t.groups, groups.data(), groups.size() * sizeof(MarchGroup)), "batch march groups");
    CK(upload(&t.queues, queues.data(), queues.size() * sizeof(MarchQueue)), "batch march queues");
    t.signature = signature_of(b, scenes, frames, g, cur, prev);
    t.valid = true;
    return IRT_OK;
}

// Launch of one pass over wave w; `rec` is the byte size of a table record.
BatchLaunch batch_launch(const irt_batch* b, size_t w, const void* table, size_t rec, int shape) {
    const uint32_t v0 = b->wave_begin[w];
    BatchLaunch B{};
    B.n = b->wave_begin[w + 1] - v0;
    B.frames = b->d_frames + v0;
    B.table = static_cast<const char*>(table) + rec * v0;
    B.gbuffer_format = b->desc.gbuffer_format;
    B.radiance_f16 = b->desc.radiance_format == IRT_RADIANCE_F16;
    B.moments_f16 = b->desc.moments_format == IRT_MOMENTS_F16;
    if (shape >= 0) {
        B.tile_start = b->d_tiles2[shape] + v0 + w;
        B.tiles = b->tiles2[shape][w];
        B.bx = kShapes[shape].bx;
        B.by = kShapes[shape].by;
    } else {
        B.tile_start = b->d_tiles1 + v0 + w;
        B.tiles = b->tiles1[w];
        B.bx = 256;
        B.by = 1;
    }
    return B;
}

// Waves for a pixel budget (0 = one wave) and their tile tables.
irt_status set_waves(irt_batch* b, uint64_t budget) {
    irt_context* ctx = b->ctx;
    b->wave_begin.assign(1, 0);
    uint64_t acc = 0;
    for (uint32_t v = 0; v < b->n; v++) {
        const uint64_t px = (uint64_t)b->W[v] * b->H[v];
        if (budget && v > b->wave_begin.back() && acc + px > budget) {
            b->wave_begin.push_back(v);
            acc = 0;
        }
        acc += px;
    }
    b->wave_begin.push_back(b->n);
    const size_t waves = b->wave_begin.size() - 1;
    std::vector<uint32_t> start(b->n + waves);
    auto build = [&](uint32_t bx, uint32_t by, std::vector<uint32_t>& tiles) {
        tiles.assign(waves, 0);
        for (size_t w = 0; w < waves; w++) {
            uint32_t t = 0;
            const uint32_t v0 = b->wave_begin[w], v1 = b->wave_begin[w + 1];
            for (uint32_t v = v0; v < v1; v++) {
                start[v + w] = t;
                t += by ? ((b->W[v] + bx - 1) / bx) * ((b->H[v] + by - 1) / by)
                        : (uint32_t)(((size_t)b->W[v] * b->H[v] + bx - 1) / bx);
            }
            start[v1 + w] = t;
            tiles[w] = t;
        }
    };
    for (int k = 0; k < kNumShapes; k++) {
        build(kShapes[k].bx, kShapes[k].by, b->tiles2[k]);
        if (b->d_tiles2[k]) cudaFree(b->d_tiles2[k]);  // the entry count follows the waves
        b->d_tiles2[k] = nullptr;
        CK(upload(&b->d_tiles2[k], start.data(), start.size() * 4), "batch tiles");
    }
    build(256, 0, b->tiles1);
    if (b->d_tiles1) cudaFree(b->d_tiles1);
    b->d_tiles1 = nullptr;
    CK(upload(&b->d_tiles1, start.data(), start.size() * 4), "batch tiles");
    b->wave_budget = budget;
    for (auto& t : b->par) free_tables(t);  // march groups follow the waves
    return IRT_OK;
}

// The frame's launches on `st`, wave after wave; `timed` records the events
// (every step's when there is one wave, else the frame's start and end).
irt_status launch_frame(irt_batch* b, int p, cudaStream_t st, const int shape_of[kNumTuned], int march_choice,
                        bool timed) {
    irt_context* ctx = b->ctx;
    ParityTables& t = b->par[p];
    const size_t waves = b->wave_begin.size() - 1;
    auto mark = [&](int k) {
        if (timed && (waves == 1 || k == 0 || k == kNumEvents - 1)) cudaEventRecord(b->ev[k], st);
    };
    const size_t la = b->la, sv = b->sv;
    mark(0);
    CK(cudaMemcpyAsync(b->d_frames, b->h_frames[p], sizeof(irt_frame) * b->n, cudaMemcpyHostToDevice, st),
       "batch frames");
    mark(1);
    for (size_t w = 0; w < waves; w++) {
        CK(irt_launch_svgf_batched(batch_launch(b, w, t.sviews[6], sv, -1),
                                   b->desc.gbuffer_format == IRT_GBUFFER_F32 ? 3 : 6, st),
           "batch guides");
        CK(irt_launch_svgf_batched(batch_launch(b, w, t.sviews[7], sv, -1), 4, st), "batch previous guides");
        mark(2);
        CK(irt_launch_lighting_batched(batch_launch(b, w, t.largs, la, -1), kStageArchive, st), "batch archive");
        mark(3);
        CK(irt_launch_lighting_batched(batch_launch(b, w, t.largs, la, shape_of[kTReuse]), kStageReuse, st),
           "batch reuse");
        mark(4);
        CK(irt_launch_lighting_batched(batch_launch(b, w, t.largs, la, shape_of[kTSpatial]), kStageSpatial, st),
           "batch spatial");
        mark(5);
        MarchBatch M{};
        M.n_groups = t.wave_groups[w + 1] - t.wave_groups[w];
        M.groups = t.groups + t.wave_groups[w];
        M.queues = t.queues;
        M.max_scene_bytes = t.max_scene_bytes;
        M.num_sms = b->num_sms;
        M.blocks_per_sm = kMarchBps[march_choice];
        M.fast = 1;
        CK(irt_launch_march_batched(M, st), "batch march");
        mark(6);
        CK(irt_launch_lighting_batched(batch_launch(b, w, t.largs, la, -1), kStageCombine, st), "batch combine");
        mark(7);
        CK(irt_launch_svgf_batched(batch_launch(b, w, t.sviews[0], sv, shape_of[kTTemporal]), 0, st),
           "batch temporal");
        mark(8);
        CK(irt_launch_svgf_batched(batch_launch(b, w, t.sviews[1], sv, shape_of[kTVariance]), 1, st),
           "batch variance");
        mark(9);
        const uint32_t iters = b->desc.settings.svgf_iterations;
        for (uint32_t i = 0; i < iters && i < 4; i++)
            CK(irt_launch_svgf_batched(batch_launch(b, w, t.sviews[2 + i], sv, shape_of[kTAtrous]), 2, st),
               "batch atrous");
        mark(10);
        CK(irt_launch_svgf_batched(batch_launch(b, w, t.history, sv, -1), 5, st), "batch history");
    }
    mark(11);
    return IRT_OK;
}

void step_ms(irt_batch* b, float ms[kNumEvents - 1]) {
    for (int k = 0; k < kNumEvents - 1; k++) cudaEventElapsedTime(&ms[k], b->ev[k], b->ev[k + 1]);
}

}  // namespace

extern "C" {

irt_status irt_batch_create(irt_context* ctx, const irt_batch_desc* desc, irt_batch** out) {
    if (!ctx || !desc || !out || desc->n_views == 0 || desc->n_views > 4096 || !desc->widths || !desc->heights)
        return IRT_E_INVALID;
    *out = nullptr;
    if (desc->settings.svgf_iterations > 4) {
        ctx->set_error("batched views run at most 4 a-trous iterations");
        return IRT_E_INVALID;
    }
    DeviceGuard dg(ctx->device);
    irt_batch* b = new (std::nothrow) irt_batch();
    if (!b) return IRT_E_NOMEM;
    b->ctx = ctx;
    b->desc = *desc;
    b->n = desc->n_views;
    b->W.assign(desc->widths, desc->widths + b->n);
    b->H.assign(desc->heights, desc->heights + b->n);
    b->desc.widths = b->W.data();
    b->desc.heights = b->H.data();
    for (uint32_t v = 0; v < b->n; v++) b->vpls.push_back(desc->vpl_counts ? desc->vpl_counts[v] : desc->settings.vpl_count);
    b->desc.vpl_counts = b->vpls.data();
    auto fail = [&](irt_status st) {
        irt_batch_destroy(b);
        return st;
    };
    for (uint32_t v = 0; v < b->n; v++) {
        irt_session_desc sd{};
        sd.settings = desc->settings;
        sd.settings.render_width = b->W[v];
        sd.settings.render_height = b->H[v];
        sd.settings.vpl_count = b->vpls[v];
        sd.gbuffer_format = desc->gbuffer_format;
        sd.radiance_format = desc->radiance_format;
        sd.moments_format = desc->moments_format;
        sd.fused = 1;
        irt_session* s = nullptr;
        irt_status st = irt_session_create(ctx, &sd, &s);
        if (st) return fail(st);
        b->sess.push_back(s);
    }
    if (cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess)
        return fail(IRT_E_CUDA);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join_out, cudaEventDisableTiming) != cudaSuccess)
        return fail(IRT_E_CUDA);
    for (int p = 0; p < 2; p++) {
        if (cudaMallocHost(&b->h_frames[p], sizeof(irt_frame) * b->n) != cudaSuccess) return fail(IRT_E_CUDA);
        if (cudaEventCreateWithFlags(&b->staged[p], cudaEventDisableTiming) != cudaSuccess) return fail(IRT_E_CUDA);
    }
    if (cudaMalloc(&b->d_frames, sizeof(irt_frame) * b->n) != cudaSuccess) return fail(IRT_E_CUDA);
    for (auto& e : b->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(IRT_E_CUDA);
    b->la = irt_lighting_args_size(desc->gbuffer_format);
    b->sv = irt_svgf_view_size(desc->gbuffer_format);
    {
        irt_status st = set_waves(b, 0);  // one wave until tuned or set
        if (st) return fail(st);
    }
    *out = b;
    return IRT_OK;
}

void irt_batch_destroy(irt_batch* b) {
    if (!b) return;
    DeviceGuard dg(b->ctx->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& t : b->par) free_tables(t);
    for (irt_session* s : b->sess) irt_session_destroy(s);
    for (int p = 0; p < 2; p++) {
        if (b->h_frames[p]) cudaFreeHost(b->h_frames[p]);
        if (b->staged[p]) cudaEventDestroy(b->staged[p]);
    }
    if (b->d_frames) cudaFree(b->d_frames);
    for (auto& e : b->ev)
        if (e) cudaEventDestroy(e);
    for (auto& p : b->d_tiles2)
        if (p) cudaFree(p);
    if (b->d_tiles1) cudaFree(b->d_tiles1);
    if (b->join_in) cudaEventDestroy(b->join_in);
    if (b->join_out) cudaEventDestroy(b->join_out);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

irt_session* irt_batch_view(irt_batch* b, uint32_t view) {
    if (!b || view >= b->n) return nullptr;
    return b->sess[view];
}

irt_status irt_batch_autotune(irt_batch* b, uint32_t frames) {
    if (!b) return IRT_E_INVALID;
    const int C = kNumShapes > kNumMarch ? kNumShapes : kNumMarch;
    b->tune_total = b->tune_left = std::max<uint32_t>(frames, (uint32_t)C);
    b->tune_ms.assign((size_t)C * (kNumTuned + 1), 0.0);
    b->tune_count.assign(C, 0);
    b->tune_wave = -1;
    for (int k = 0; k < kNumWaves; k++) b->wave_ms[k] = 0.0, b->wave_count[k] = 0;
    return set_waves(b, 0);  // shapes are timed per pass on one wave
}

irt_status irt_batch_tuning(const irt_batch* b, char* out, size_t len) {
    if (!b || !out || len == 0) return IRT_E_INVALID;
    std::string s;
    for (int k = 0; k < kNumTuned; k++) {
        char buf[48];
        std::snprintf(buf, sizeof(buf), "%s=%ux%u ", kTunedNames[k], kShapes[b->shape_of[k]].bx,
                      kShapes[b->shape_of[k]].by);
        s += buf;
    }
    const int bps = kMarchBps[b->march_choice];
    s += "march_ctas_per_sm=" + (bps ? std::to_string(bps) : std::string("max"));
    s += " waves=" + std::to_string(b->wave_begin.size() - 1) + " wave_budget_px=" +
         (b->wave_budget ? std::to_string(b->wave_budget) : std::string("all"));
    std::snprintf(out, len, "%s", s.c_str());
    return IRT_OK;
}

irt_status irt_batch_set_waves(irt_batch* b, uint64_t budget_px) {
    if (!b) return IRT_E_INVALID;
    irt_context* ctx = b->ctx;
    DeviceGuard dg(ctx->device);
    CK(cudaStreamSynchronize(b->stream), "batch waves");
    b->tune_wave = -1;
    return set_waves(b, budget_px);
}

irt_status irt_batch_pass_ms(irt_batch* b, float* out12) {
    if (!b || !out12) return IRT_E_INVALID;
    irt_context* ctx = b->ctx;
    if (b->timed_pending && b->wave_begin.size() > 2) {  // several waves: the frame's total only
        CK(cudaEventSynchronize(b->ev[kNumEvents - 1]), "batch pass timing");
        float total = 0.f;
        cudaEventElapsedTime(&total, b->ev[0], b->ev[kNumEvents - 1]);
        for (float& v : b->pass_ms) v = 0.f;
        b->pass_ms[kPTotal] = total;
        b->timed_pending = false;
    }
    if (b->timed_pending) {
        CK(cudaEventSynchronize(b->ev[kNumEvents - 1]), "batch pass timing");
        float ms[kNumEvents - 1];
        step_ms(b, ms);
        const int slot[kNumEvents - 1] = {-1, kPGuides, kPArchive, kPReuse, kPSpatial, kPMarch, kPCombine,
                                          kPTemporal, kPVariance, kPAtrous, kPHistory};
        float total = 0.f;
        for (int k = 0; k < kNumEvents - 1; k++) {
            if (slot[k] >= 0) b->pass_ms[slot[k]] = ms[k];
            total += ms[k];
        }
        b->pass_ms[kPTotal] = total;
        b->timed_pending = false;
    }
    std::memcpy(out12, b->pass_ms, sizeof(b->pass_ms));
    return IRT_OK;
}

irt_status irt_batch_render(irt_batch* b, irt_scene* const* scenes, const irt_frame* frames, const irt_gbuffer* g,
                            const irt_vpl* const* cur, const irt_vpl* const* prev, void* stream) {
    if (!b || !scenes || !frames || !g || !cur || !prev) return IRT_E_INVALID;
    irt_context* ctx = b->ctx;
    DeviceGuard dg(ctx->device);
    cudaStream_t caller = static_cast<cudaStream_t>(stream);
    cudaStream_t st = b->stream;
    const uint32_t index = frames[0].size[2];
    const irt_settings& set = b->desc.settings;
    for (uint32_t v = 0; v < b->n; v++) {
        const irt_frame& f = frames[v];
        const irt_scene* sc = scenes[v];
        if (!sc || !cur[v] || !prev[v]) return IRT_E_INVALID;
        if (f.size[0] != b->W[v] || f.size[1] != b->H[v] || f.size[2] != index) {
            ctx->set_error("batched frame size or index differs from the batch's");
            return IRT_E_INVALID;
        }
        if (f.flags[2] != 0u) {
            ctx->set_error("debug views are not batched");
            return IRT_E_INVALID;
        }
        if (f.counts[1] != b->vpls[v] || f.counts[3] != sc->object_count || f.counts[0] > sc->light_count ||
            (uint32_t)f.rr[2] != set.restir_max_history) {
            ctx->set_error("batched frame counts differ from the batch/scene");
            return IRT_E_INVALID;
        }
        if (f.restir[0] == 0 || f.restir[0] > 256 || f.restir[1] == 0 || f.restir[1] > 256 || f.restir[2] > 32 ||
            f.restir[3] > 256 || !(f.sdf[0] >= 1.f && f.sdf[0] <= 1024.f) || !(f.sdf[1] > 0.f)) {
            ctx->set_error("frame ReSTIR/SDF parameters out of range");
            return IRT_E_INVALID;
        }
        if (g[v].format != b->desc.gbuffer_format || !g[v].depth || !g[v].normal || !g[v].color || !g[v].params ||
            !g[v].motion) {
            ctx->set_error("G-buffer format or planes invalid");
            return IRT_E_INVALID;
        }
    }
    const int p = (int)(index % 2u);
    ParityTables& t = b->par[p];
    if (!t.valid || t.signature != signature_of(b, scenes, frames, g, cur, prev)) {
        CK(cudaStreamSynchronize(st), "batch tables");  // tables in use by queued work
        irt_status rc = build_tables(b, p, scenes, frames, g, cur, prev);
        if (rc) return rc;
    }
    // The pinned frame staging of this parity is free once its last use ran.
    CK(cudaEventSynchronize(b->staged[p]), "batch staging");
    std::memcpy(b->h_frames[p], frames, sizeof(irt_frame) * b->n);
    // Work on the batch stream follows everything queued on the caller's.
    CK(cudaEventRecord(b->join_in, caller), "batch join");
    CK(cudaStreamWaitEvent(st, b->join_in, 0), "batch join");
    bool next_waves = false;
    int waves_to = 0;
    if (b->tune_left > 0) {
        // Phase 1: every candidate shape for all tuned passes (one wave).
        const int C = (int)b->tune_count.size();
        const int c = (int)((b->tune_total - b->tune_left) % (uint32_t)C);
        int shapes[kNumTuned];
        for (int k = 0; k < kNumTuned; k++) shapes[k] = c % kNumShapes;
        irt_status rc = launch_frame(b, p, st, shapes, c % kNumMarch, true);
        if (rc) return rc;
        CK(cudaEventSynchronize(b->ev[kNumEvents - 1]), "batch tuning");
        float ms[kNumEvents - 1];
        step_ms(b, ms);
        const int slot[kNumTuned] = {3, 4, 7, 8, 9};  // reuse, spatial, temporal, variance, a-trous steps
        double* row = &b->tune_ms[(size_t)c * (kNumTuned + 1)];
        for (int k = 0; k < kNumTuned; k++) row[k] += ms[slot[k]];
        row[kNumTuned] += ms[5];  // march
        b->tune_count[c]++;
        if (--b->tune_left == 0) {
            for (int k = 0; k < kNumTuned; k++) {
                int best = 0;
                double best_ms = 1e30;
                for (int cc = 0; cc < kNumShapes && cc < C; cc++) {
                    if (!b->tune_count[cc]) continue;
                    double m = b->tune_ms[(size_t)cc * (kNumTuned + 1) + k] / b->tune_count[cc];
                    if (m < best_ms) best_ms = m, best = cc;
                }
                b->shape_of[k] = best;
            }
            // The march is tuned over its own candidates: mean time per choice.
            double sum[kNumMarch] = {0, 0, 0};
            int cnt[kNumMarch] = {0, 0, 0};
            for (int cc = 0; cc < C; cc++) {
                if (!b->tune_count[cc]) continue;
                sum[cc % kNumMarch] += b->tune_ms[(size_t)cc * (kNumTuned + 1) + kNumTuned];
                cnt[cc % kNumMarch] += b->tune_count[cc];
            }
            int best = 0;
            for (int k = 1; k < kNumMarch; k++)
                if (cnt[k] && (!cnt[best] || sum[k] / cnt[k] < sum[best] / cnt[best])) best = k;
            b->march_choice = best;
            b->tune_wave = 0;  // phase 2 starts with one wave (the tables in use)
        }
        b->pass_ms[kPGraph] = 0.f;
    } else if (b->tune_wave >= 0) {
        // Phase 2: each wave budget with the chosen shapes, timed per frame.
        irt_status rc = launch_frame(b, p, st, b->shape_of, b->march_choice, true);
        if (rc) return rc;
        CK(cudaEventSynchronize(b->ev[kNumEvents - 1]), "batch tuning");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->ev[0], b->ev[kNumEvents - 1]);
        b->wave_ms[b->tune_wave] += ms;
        b->wave_count[b->tune_wave]++;
        next_waves = true;
        if (b->tune_wave + 1 < kNumWaves) {
            waves_to = ++b->tune_wave;
        } else {
            int best = 0;
            for (int k = 1; k < kNumWaves; k++)
                if (b->wave_count[k] && b->wave_ms[k] / b->wave_count[k] < b->wave_ms[best] / b->wave_count[best])
                    best = k;
            waves_to = best;
            b->tune_wave = -1;
        }
        b->pass_ms[kPGraph] = 0.f;
    } else if (b->desc.use_graphs && t.graph) {
        CK(cudaGraphLaunch(t.graph, st), "batch graph launch");
        b->pass_ms[kPGraph] = 1.f;
    } else if (b->desc.use_graphs && t.renders >= 1) {
        // Capture this parity's launch sequence once and replay it from now on
        // (after one direct render, which sets every kernel attribute).
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "batch capture");
        irt_status rc = launch_frame(b, p, st, b->shape_of, b->march_choice, false);
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        CK(e, "batch capture end");
        e = cudaGraphInstantiate(&t.graph, graph, 0);
        cudaGraphDestroy(graph);
        CK(e, "batch graph instantiate");
        CK(cudaGraphLaunch(t.graph, st), "batch graph launch");
        b->pass_ms[kPGraph] = 1.f;
    } else {
        irt_status rc = launch_frame(b, p, st, b->shape_of, b->march_choice, true);
        if (rc) return rc;
        t.renders++;
        b->timed_pending = true;  // read (with a sync) only when asked for
        b->pass_ms[kPGraph] = 0.f;
    }
    if (next_waves) {  // the next frame runs the next wave budget (tables rebuilt then)
        CK(cudaStreamSynchronize(st), "batch tuning");
        irt_status rc = set_waves(b, kWavePx[waves_to]);
        if (rc) return rc;
    }
    CK(cudaEventRecord(b->staged[p], st), "batch staging event");
    CK(cudaEventRecord(b->join_out, st), "batch join");
    CK(cudaStreamWaitEvent(caller, b->join_out, 0), "batch join");
    for (uint32_t v = 0; v < b->n; v++) {
        irt_session* s = b->sess[v];
        s->last_frame = index;
        s->have_frame = true;
        s->guide_frame = index;
    }
    return IRT_OK;
}

}  // extern "C"
