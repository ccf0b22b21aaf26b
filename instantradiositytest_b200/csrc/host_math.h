// host_math.h — small host-side matrix/vector helpers (column-major mat4 like
// glam::Mat4).  Matrices are composed in double and stored as f32; the device
// kernels and the CPU oracle both consume the stored f32 bytes.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/irt.h"

namespace irt {

struct D3 {
    double x, y, z;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double length(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 normalize(D3 a) { return a * (1.0 / length(a)); }

struct M4 {  // column-major, m[c][r]
    double m[4][4];
};
inline M4 identity() {
    M4 r{};
    for (int i = 0; i < 4; i++) r.m[i][i] = 1.0;
    return r;
}
inline M4 mul(const M4& a, const M4& b) {
    M4 r{};
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) {
            double s = 0;
            for (int k = 0; k < 4; k++) s += a.m[k][rr] * b.m[c][k];
            r.m[c][rr] = s;
        }
    return r;
}
inline M4 from_f32(const irt_mat4& a) {
    M4 r;
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) r.m[c][rr] = a.m[c * 4 + rr];
    return r;
}
inline irt_mat4 to_f32(const M4& a) {
    irt_mat4 r;
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) r.m[c * 4 + rr] = (float)a.m[c][rr];
    return r;
}
// General 4x4 inverse (cofactor expansion).
inline M4 inverse(const M4& a) {
    double m[16], inv[16];
    for (int c = 0; c < 4; c++)
        for (int r = 0; r < 4; r++) m[c * 4 + r] = a.m[c][r];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
             m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
             m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
             m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
              m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
             m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
             m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
             m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
              m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
             m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
             m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
              m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
              m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
             m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
             m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
              m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
              m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    double id = det != 0.0 ? 1.0 / det : 0.0;
    M4 r;
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) r.m[c][rr] = inv[c * 4 + rr] * id;
    return r;
}
inline void transform(const M4& a, double x, double y, double z, double w, double out[4]) {
    for (int r = 0; r < 4; r++) out[r] = a.m[0][r] * x + a.m[1][r] * y + a.m[2][r] * z + a.m[3][r] * w;
}
// Mat4::from_scale_rotation_translation (src/scene.rs:18-25) from a unit
// quaternion (x, y, z, w).
inline M4 scale_rotation_translation(double s, const double q[4], D3 t) {
    double x = q[0], y = q[1], z = q[2], w = q[3];
    double n = std::sqrt(x * x + y * y + z * z + w * w);
    x /= n;
    y /= n;
    z /= n;
    w /= n;
    M4 r{};
    r.m[0][0] = (1 - 2 * (y * y + z * z)) * s;
    r.m[0][1] = (2 * (x * y + w * z)) * s;
    r.m[0][2] = (2 * (x * z - w * y)) * s;
    r.m[1][0] = (2 * (x * y - w * z)) * s;
    r.m[1][1] = (1 - 2 * (x * x + z * z)) * s;
    r.m[1][2] = (2 * (y * z + w * x)) * s;
    r.m[2][0] = (2 * (x * z + w * y)) * s;
    r.m[2][1] = (2 * (y * z - w * x)) * s;
    r.m[2][2] = (1 - 2 * (x * x + y * y)) * s;
    r.m[3][0] = t.x;
    r.m[3][1] = t.y;
    r.m[3][2] = t.z;
    r.m[3][3] = 1;
    return r;
}
// Right-handed perspective with [0,1] depth (DirectX convention), the
// projection of Camera::matrix (src/scene.rs:117-126).
inline M4 perspective_rh_zo(double fov_y, double aspect, double near, double far) {
    double h = std::cos(0.5 * fov_y) / std::sin(0.5 * fov_y);
    double w = h / aspect;
    double r = far / (near - far);
    M4 m{};
    m.m[0][0] = w;
    m.m[1][1] = h;
    m.m[2][2] = r;
    m.m[2][3] = -1;
    m.m[3][2] = r * near;
    return m;
}
// World-to-camera transform of a camera at `eye` looking at `target` with
// world up `up` (camera looks down its -Z).
inline M4 look_at_rh(D3 eye, D3 target, D3 up) {
    D3 f = normalize(target - eye);
    D3 s = normalize(cross(f, up));
    D3 u = cross(s, f);
    M4 m = identity();
    m.m[0][0] = s.x;
    m.m[1][0] = s.y;
    m.m[2][0] = s.z;
    m.m[0][1] = u.x;
    m.m[1][1] = u.y;
    m.m[2][1] = u.z;
    m.m[0][2] = -f.x;
    m.m[1][2] = -f.y;
    m.m[2][2] = -f.z;
    m.m[3][0] = -dot(s, eye);
    m.m[3][1] = -dot(u, eye);
    m.m[3][2] = dot(f, eye);
    return m;
}

inline uint32_t f32_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

}  // namespace irt
