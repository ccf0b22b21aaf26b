// dev_prims.cuh — f32 ray casts against the flattened analytic primitive
// table of a synthetic workload (boxes and spheres in object space).  Used by
// the CUDA G-buffer producer (primary rays) and the CUDA VPL generator (the
// stand-in for the ray query of vpl.wgsl).
#pragma once
#include <cuda_runtime.h>

#include "workload.h"

namespace irtd {

__device__ __forceinline__ void xf4(const float* m, float x, float y, float z, float w, float o[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) o[r] = m[r] * x + m[4 + r] * y + m[8 + r] * z + m[12 + r] * w;
}

// Nearest front entry t in (tmin, tmax) along o + t d over all primitives:
// slab test for boxes (an origin inside a box is no hit), nearest root for
// spheres.  Returns the primitive index or -1, with t and the object-space
// normal of the entered face in nl.
__device__ __forceinline__ int cast_prims(const irt::GPrim* prims, uint32_t n_prims, const float o[3],
                                          const float d[3], float tmin, float tmax, float& t_out, float nl[3]) {
    float best = tmax;
    int hit = -1;
    for (uint32_t k = 0; k < n_prims; k++) {
        const irt::GPrim& p = prims[k];
        float lo4[4], ld4[4];
        xf4(p.inv_model, o[0], o[1], o[2], 1.f, lo4);
        xf4(p.inv_model, d[0], d[1], d[2], 0.f, ld4);
        float t = 0.f;
        float nn[3] = {0, 0, 0};
        bool h = false;
        if (p.sphere) {
            float r = p.lo[0];
            float b = lo4[0] * ld4[0] + lo4[1] * ld4[1] + lo4[2] * ld4[2];
            float a = ld4[0] * ld4[0] + ld4[1] * ld4[1] + ld4[2] * ld4[2];
            float c = lo4[0] * lo4[0] + lo4[1] * lo4[1] + lo4[2] * lo4[2] - r * r;
            float disc = b * b - a * c;
            if (disc >= 0.f) {
                t = (-b - sqrtf(disc)) / a;
                if (t >= tmin && t < best) {
                    h = true;
                    for (int q = 0; q < 3; q++) nn[q] = (lo4[q] + ld4[q] * t) / r;
                }
            }
        } else {
            float t0 = tmin, t1 = best;
            int axis = -1;
            float sign = 0.f;
            bool miss = false;
            for (int a = 0; a < 3 && !miss; a++) {
                float inv = 1.f / ld4[a];
                float ta = (p.lo[a] - lo4[a]) * inv, tb = (p.hi[a] - lo4[a]) * inv;
                float s = -1.f;
                if (ta > tb) {
                    float tmp = ta;
                    ta = tb;
                    tb = tmp;
                    s = 1.f;
                }
                if (ta > t0) {
                    t0 = ta;
                    axis = a;
                    sign = s;
                }
                t1 = fminf(t1, tb);
                if (t0 > t1) miss = true;
            }
            if (!miss && axis >= 0 && t0 < best) {
                h = true;
                t = t0;
                nn[axis] = sign;
            }
        }
        if (h) {
            best = t;
            hit = (int)k;
            nl[0] = nn[0];
            nl[1] = nn[1];
            nl[2] = nn[2];
        }
    }
    t_out = best;
    return hit;
}

}  // namespace irtd
