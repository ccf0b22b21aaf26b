// server.cpp — render server: continuous batching of render sessions over
// one context (irt_server_* in irt.h).
//
// One host thread drives the loop: admit arrived requests in arrival order
// while their bytes fit the budget and a slot is free, launch the next frame
// of every admitted session that is due (at most two in flight per session),
// observe completions through CUDA events, retire finished sessions (their
// history and inputs are freed and the bytes return to the budget).
// Sessions are spread over a fixed set of CUDA streams, so frames of
// different sessions run concurrently on the device.  Completion times are
// device timestamps (cudaEventElapsedTime against a base event) mapped onto
// the host clock.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/irt.h"
#include "workload.h"

namespace {

using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

uint64_t gbuffer_bytes_per_pixel(int32_t fmt) {
    switch (fmt) {
    case IRT_GBUFFER_F32: return 4 + 16 + 16 + 8 + 8;
    case IRT_GBUFFER_F16: return 4 + 8 + 8 + 4 + 4;
    default: return 4 + 4 + 4 + 4 + 4;
    }
}

struct Inflight {
    uint32_t frame = 0;
    double due = 0;
    cudaEvent_t start = nullptr, end = nullptr;
    bool capture = false;
};

struct Active {
    irt_request req{};
    irt_scene* scene = nullptr;
    irt_session* session = nullptr;
    cudaStream_t stream = nullptr;
    void* gbuf = nullptr;  // the five planes in one allocation
    irt_gbuffer g{};
    irt_vpl* vpls = nullptr;  // pools [0], [1] and a zero pool [2]
    void* staging = nullptr;  // pinned host copy of the captured frame
    uint64_t capture_bytes = 0;
    uint64_t bytes = 0;
    uint32_t W = 0, H = 0, vpl_count = 0;
    uint32_t next_frame = 0;
    double admitted = 0, last_done = 0;
    std::vector<irt_object> objects;
    std::vector<irt_node> nodes;
    std::vector<irt_light> lights;
    irt_frame frame{};
    Inflight fl[2];
    uint32_t inflight = 0, head = 0;  // ring of in-flight frames
    cudaEvent_t ev_pool[4] = {nullptr, nullptr, nullptr, nullptr};
};

float percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.f;
    std::sort(v.begin(), v.end());
    size_t k = (size_t)std::min<double>(v.size() - 1, std::max(0.0, q * (v.size() - 1) + 0.5));
    return v[k];
}

}  // namespace

struct irt_server {
    irt_context* ctx = nullptr;
    irt_server_desc d{};
    std::vector<cudaStream_t> streams;
    cudaStream_t control = nullptr;  // idle stream for reads of finished sessions
    std::deque<irt_request> queue;
    std::string error;
};

static irt_session_desc session_desc_for(const irt_server* s, const irt_workload* wl) {
    irt_session_desc sd{};
    irt_workload_settings(wl, &sd.settings);
    sd.gbuffer_format = s->d.gbuffer_format;
    sd.radiance_format = s->d.radiance_format;
    sd.moments_format = s->d.moments_format;
    sd.fused = s->d.fused;
    sd.keep_candidates = 0;
    sd.exact_march = 0;
    return sd;
}

extern "C" uint64_t irt_server_request_bytes(const irt_server* s, const irt_request* r) {
    if (!s || !r || !r->workload) return 0;
    const irt::Workload& w = r->workload->w;
    irt_session_desc sd = session_desc_for(s, r->workload);
    const uint64_t P = (uint64_t)w.spec.width * w.spec.height;
    const uint64_t n = w.objs.size();
    const uint64_t texel = w.spec.sdf_format == IRT_SDF_F16 ? 2 : 4;
    const uint64_t atlas = (uint64_t)w.atlas_dims[0] * w.atlas_dims[1] * w.atlas_dims[2] * texel;
    uint64_t scene = atlas + atlas / 8 + (4u << 20);                 // atlas (+ array padding), leaf cache
    scene += n * (208 + 2 * 48 + 176 + 33ull * 33 * 33 * 4) + 128 * w.meshes.size() + 2 * 48 * w.lights.size();
    for (const irt_mesh& m : w.meshes)  // corner cells of the field meshes (8 texels per cell)
        if (m.geometry_lo[3] <= .5f) scene += (uint64_t)(m.field[3] - 1) * (m.field[3] - 1) * (m.field[3] - 1) * texel * 8;
    const uint64_t inputs = P * gbuffer_bytes_per_pixel(s->d.gbuffer_format) + 3ull * sd.settings.vpl_count * 48;
    return irt_session_bytes(&sd) + scene + inputs;
}

extern "C" irt_status irt_server_create(irt_context* ctx, const irt_server_desc* desc, irt_server** out) {
    if (!ctx || !desc || !out) return IRT_E_INVALID;
    *out = nullptr;
    if (desc->streams == 0 || desc->streams > 64 || desc->frame_rate < 0.f || desc->hbm_budget_bytes == 0)
        return IRT_E_INVALID;
    auto* s = new (std::nothrow) irt_server();
    if (!s) return IRT_E_NOMEM;
    s->ctx = ctx;
    s->d = *desc;
    for (uint32_t i = 0; i < desc->streams; i++) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            irt_server_destroy(s);
            return IRT_E_CUDA;
        }
        s->streams.push_back(st);
    }
    if (cudaStreamCreateWithFlags(&s->control, cudaStreamNonBlocking) != cudaSuccess) {
        irt_server_destroy(s);
        return IRT_E_CUDA;
    }
    *out = s;
    return IRT_OK;
}

extern "C" void irt_server_destroy(irt_server* s) {
    if (!s) return;
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->control) cudaStreamDestroy(s->control);
    delete s;
}

extern "C" irt_status irt_server_submit(irt_server* s, const irt_request* r) {
    if (!s || !r || !r->workload || r->frames == 0 || !(r->arrival_s >= 0.0)) return IRT_E_INVALID;
    if (r->times) r->times[0] = r->times[1] = r->times[2] = -1.0;
    // keep the queue ordered by arrival (stable for equal times)
    auto it = std::upper_bound(s->queue.begin(), s->queue.end(), *r,
                               [](const irt_request& a, const irt_request& b) { return a.arrival_s < b.arrival_s; });
    s->queue.insert(it, *r);
    return IRT_OK;
}

// Frees a session whose frames have all completed (or, on an error path,
// after the device was synchronised).
static void release(Active* a) {
    for (cudaEvent_t e : a->ev_pool)
        if (e) cudaEventDestroy(e);
    if (a->session) irt_session_destroy(a->session);
    if (a->scene) irt_scene_destroy(a->scene);
    if (a->gbuf) cudaFree(a->gbuf);
    if (a->vpls) cudaFree(a->vpls);
    if (a->staging) cudaFreeHost(a->staging);
    delete a;
}

static irt_status admit(irt_server* s, const irt_request& r, cudaStream_t st, Active** out) {
    auto* a = new (std::nothrow) Active();
    if (!a) return IRT_E_NOMEM;
    a->req = r;
    a->stream = st;
    irt::Workload& w = r.workload->w;
    a->W = w.spec.width;
    a->H = w.spec.height;
    irt_session_desc sd = session_desc_for(s, r.workload);
    a->vpl_count = sd.settings.vpl_count;
    const void* atlas = w.spec.sdf_format == IRT_SDF_F16 ? (const void*)w.atlas16.data() : (const void*)w.atlas32.data();
    irt_status rc = irt_scene_create(s->ctx, w.meshes.data(), (uint32_t)w.meshes.size(), atlas, w.atlas_dims,
                                     w.spec.sdf_format, &a->scene);
    if (!rc) rc = irt_session_create(s->ctx, &sd, &a->session);
    const size_t P = (size_t)a->W * a->H;
    const uint64_t gb = P * gbuffer_bytes_per_pixel(s->d.gbuffer_format);
    if (!rc && cudaMalloc(&a->gbuf, gb) != cudaSuccess) rc = IRT_E_CUDA;
    if (!rc && cudaMalloc(&a->vpls, 3ull * a->vpl_count * sizeof(irt_vpl)) != cudaSuccess) rc = IRT_E_CUDA;
    if (!rc && cudaMemsetAsync(a->vpls + 2ull * a->vpl_count, 0, a->vpl_count * sizeof(irt_vpl), st) != cudaSuccess)
        rc = IRT_E_CUDA;
    for (int k = 0; k < 4 && !rc; k++)
        if (cudaEventCreate(&a->ev_pool[k]) != cudaSuccess) rc = IRT_E_CUDA;
    if (!rc && r.capture) {
        void* p;
        uint64_t b;
        if (irt_session_buffer(a->session, IRT_BUF_FILTERED, &p, &b) != IRT_OK ||
            cudaMallocHost(&a->staging, b) != cudaSuccess)
            rc = IRT_E_CUDA;
        a->capture_bytes = b;
    }
    if (rc) {
        release(a);
        return rc;
    }
    // Plane layout: depth f32, then normal, color, params, motion.
    char* base = static_cast<char*>(a->gbuf);
    uint64_t nb, cb, pb, mb;
    switch (s->d.gbuffer_format) {
    case IRT_GBUFFER_F32: nb = 16, cb = 16, pb = 8, mb = 8; break;
    case IRT_GBUFFER_F16: nb = 8, cb = 8, pb = 4, mb = 4; break;
    default: nb = 4, cb = 4, pb = 4, mb = 4; break;
    }
    a->g.format = s->d.gbuffer_format;
    a->g.depth = reinterpret_cast<const float*>(base);
    a->g.normal = base + P * 4;
    a->g.color = base + P * (4 + nb);
    a->g.params = base + P * (4 + nb + cb);
    a->g.motion = base + P * (4 + nb + cb + pb);
    (void)mb;
    a->objects.resize(w.objs.size());
    a->nodes.resize(2 * w.objs.size() - 1);
    a->lights.resize(std::max<size_t>(w.lights.size(), 1));
    *out = a;
    return IRT_OK;
}

// One frame of a session on its stream: scene data, G-buffer, VPL pool, the
// lighting + SVGF hot path, and (for the capture frame) the output copy.
static irt_status launch_frame(irt_server* s, Active* a, double due) {
    irt::Workload& w = a->req.workload->w;
    const uint32_t k = a->next_frame;
    Inflight& fl = a->fl[(a->head + a->inflight) % 2];
    fl.frame = k;
    fl.due = due;
    fl.start = a->ev_pool[((a->head + a->inflight) % 2) * 2];
    fl.end = a->ev_pool[((a->head + a->inflight) % 2) * 2 + 1];
    fl.capture = a->req.capture && k == a->req.capture_frame;
    cudaEventRecord(fl.start, a->stream);
    w.frame_data(k, 0, &a->frame, a->objects.data(), a->nodes.data(), a->lights.data());
    const uint32_t nl = (uint32_t)w.lights.size();
    irt_status rc = irt_scene_update(a->scene, a->objects.data(), (uint32_t)a->objects.size(), a->nodes.data(),
                                     (uint32_t)a->nodes.size(), nl ? a->lights.data() : nullptr, nl, a->stream);
    if (rc) return rc;
    rc = irt_gbuffer_render(s->ctx, a->req.workload, &a->frame, nullptr, a->g.format, const_cast<float*>(a->g.depth),
                            const_cast<void*>(a->g.normal), const_cast<void*>(a->g.color),
                            const_cast<void*>(a->g.params), const_cast<void*>(a->g.motion), a->stream);
    if (rc) return rc;
    irt_vpl* cur = a->vpls + (size_t)(k % 2) * a->vpl_count;
    const irt_vpl* prev = k == 0 ? a->vpls + 2ull * a->vpl_count : a->vpls + (size_t)((k + 1) % 2) * a->vpl_count;
    rc = irt_vpl_generate(a->scene, a->req.workload, &a->frame, cur, a->stream);
    if (rc) return rc;
    rc = irt_render_frame(a->session, a->scene, &a->frame, &a->g, cur, prev, a->stream);
    if (rc) return rc;
    if (fl.capture) {
        void* p;
        uint64_t b;
        irt_session_buffer(a->session, IRT_BUF_FILTERED, &p, &b);
        if (cudaMemcpyAsync(a->staging, p, b, cudaMemcpyDeviceToHost, a->stream) != cudaSuccess) return IRT_E_CUDA;
    }
    if (cudaEventRecord(fl.end, a->stream) != cudaSuccess) return IRT_E_CUDA;
    a->inflight++;
    a->next_frame++;
    return IRT_OK;
}

extern "C" irt_status irt_server_run(irt_server* s, irt_server_stats* stats) {
    if (!s || !stats) return IRT_E_INVALID;
    std::memset(stats, 0, sizeof(*stats));
    std::vector<float> latency, frame_ms, wait;
    std::vector<Active*> active;
    uint64_t admitted_bytes = 0, peak_bytes = 0;
    uint64_t sessions = 0, rejected = 0, frames = 0;
    double pixel_frames = 0, active_time = 0, peak_active = 0;
    double first_admit = -1, last_done = 0;
    uint32_t next_stream = 0;
    irt_status rc = IRT_OK;

    cudaEvent_t base;
    if (cudaEventCreate(&base) != cudaSuccess) return IRT_E_CUDA;
    cudaEventRecord(base, s->streams[0]);
    cudaEventSynchronize(base);
    const Clock::time_point t0 = Clock::now();
    double last_t = 0;

    while (!rc && (!s->queue.empty() || !active.empty())) {
        bool progressed = false;
        // completions
        for (size_t i = 0; i < active.size();) {
            Active* a = active[i];
            while (a->inflight) {
                Inflight& fl = a->fl[a->head];
                cudaError_t q = cudaEventQuery(fl.end);
                if (q == cudaErrorNotReady) break;
                if (q != cudaSuccess) {
                    rc = IRT_E_CUDA;
                    break;
                }
                float ms_done = 0, ms_frame = 0;
                cudaEventElapsedTime(&ms_done, base, fl.end);
                cudaEventElapsedTime(&ms_frame, fl.start, fl.end);
                const double done = ms_done / 1000.0;
                latency.push_back((float)((done - fl.due) * 1000.0));
                frame_ms.push_back(ms_frame);
                last_done = std::max(last_done, done);
                a->last_done = std::max(a->last_done, done);
                frames++;
                pixel_frames += (double)a->W * a->H;
                if (fl.capture) std::memcpy(a->req.capture, a->staging, a->capture_bytes);
                a->head = (a->head + 1) % 2;
                a->inflight--;
                progressed = true;
            }
            if (rc) break;
            if (a->inflight == 0 && a->next_frame >= a->req.frames) {
                // All of the session's work has completed: read its error
                // word on the idle control stream, not behind other sessions.
                if (irt_session_check(a->session, s->control) != IRT_OK) rc = IRT_E_DEVICE;
                if (a->req.times) {
                    a->req.times[0] = a->admitted;
                    a->req.times[1] = a->last_done;
                    a->req.times[2] = seconds_since(t0);
                }
                admitted_bytes -= a->bytes;
                release(a);
                active.erase(active.begin() + (long)i);
                progressed = true;
                continue;
            }
            i++;
        }
        if (rc) break;
        double now = seconds_since(t0);
        // admissions, in arrival order
        while (!s->queue.empty() && s->queue.front().arrival_s <= now) {
            const irt_request& r = s->queue.front();
            const uint64_t need = irt_server_request_bytes(s, &r);
            if (need > s->d.hbm_budget_bytes) {
                rejected++;
                s->queue.pop_front();
                continue;
            }
            if (admitted_bytes + need > s->d.hbm_budget_bytes ||
                (s->d.max_sessions && active.size() >= s->d.max_sessions))
                break;
            Active* a = nullptr;
            cudaStream_t st = s->streams[next_stream++ % s->streams.size()];
            irt_status ar = admit(s, r, st, &a);
            if (ar == IRT_E_ADMISSION) break;  // the context's own budget: wait for retirements
            if (ar) {
                rc = ar;
                break;
            }
            now = seconds_since(t0);
            a->admitted = now;
            a->bytes = need;
            admitted_bytes += need;
            peak_bytes = std::max(peak_bytes, admitted_bytes);
            wait.push_back((float)((now - r.arrival_s) * 1000.0));
            if (first_admit < 0) first_admit = now;
            sessions++;
            active.push_back(a);
            s->queue.pop_front();
            progressed = true;
        }
        if (rc) break;
        // launches: every session gets its due frames, up to two in flight;
        // a session behind schedule gets both back to back on its stream, so
        // consecutive kernels reuse its scene and history in L2.
        now = seconds_since(t0);
        for (Active* a : active) {
            while (a->inflight < 2 && a->next_frame < a->req.frames) {
                double due = s->d.frame_rate > 0.f ? a->admitted + a->next_frame / (double)s->d.frame_rate : now;
                if (due > now) break;
                rc = launch_frame(s, a, due);
                if (rc) break;
                progressed = true;
            }
            if (rc) break;
        }
        now = seconds_since(t0);
        active_time += active.size() * (now - last_t);
        last_t = now;
        peak_active = std::max(peak_active, (double)active.size());
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    if (!active.empty()) cudaDeviceSynchronize();
    for (Active* a : active) release(a);
    cudaEventDestroy(base);
    const double span = last_done - std::max(first_admit, 0.0);
    stats->frames = frames;
    stats->sessions = sessions;
    stats->rejected = rejected;
    stats->pixel_frames = pixel_frames;
    stats->seconds = span;
    stats->mpix_frames_per_s = span > 0 ? pixel_frames / span / 1e6 : 0;
    stats->p50_latency_ms = percentile(latency, .5);
    stats->p99_latency_ms = percentile(latency, .99);
    stats->p50_frame_ms = percentile(frame_ms, .5);
    stats->p99_frame_ms = percentile(frame_ms, .99);
    stats->p50_wait_ms = percentile(wait, .5);
    stats->p99_wait_ms = percentile(wait, .99);
    stats->mean_active = last_t > 0 ? (float)(active_time / last_t) : 0.f;
    stats->peak_active = (float)peak_active;
    stats->peak_bytes = peak_bytes;
    return rc;
}
