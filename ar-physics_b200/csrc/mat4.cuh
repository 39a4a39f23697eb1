// mat4.cuh -- column-major 4x4 float matrices with GLSL product conventions,
// for the per-particle strain/stress math of the solid kernels.
#pragma once

#include <cuda_runtime.h>

namespace arp {

struct M4 {
    float m[4][4];  // m[column][row]
};

__host__ __device__ __forceinline__ M4 m4_zero() {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = 0.0f;
    return r;
}
__host__ __device__ __forceinline__ M4 m4_ident() {
    M4 r = m4_zero();
#pragma unroll
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
}
__host__ __device__ __forceinline__ M4 m4_add(const M4& a, const M4& b) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = a.m[c][k] + b.m[c][k];
    return r;
}
__host__ __device__ __forceinline__ M4 m4_sub(const M4& a, const M4& b) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = a.m[c][k] - b.m[c][k];
    return r;
}
__host__ __device__ __forceinline__ M4 m4_scale(float s, const M4& a) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = s * a.m[c][k];
    return r;
}
__host__ __device__ __forceinline__ M4 m4_div(const M4& a, float s) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = a.m[c][k] / s;
    return r;
}
__host__ __device__ __forceinline__ M4 m4_mul(const M4& a, const M4& b) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            r.m[c][k] = ((a.m[0][k] * b.m[c][0] + a.m[1][k] * b.m[c][1]) + a.m[2][k] * b.m[c][2]) + a.m[3][k] * b.m[c][3];
    return r;
}
__host__ __device__ __forceinline__ M4 m4_transpose(const M4& a) {
    M4 r;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) r.m[c][k] = a.m[k][c];
    return r;
}
__host__ __device__ __forceinline__ float m4_dot(const M4& x, const M4& y) {
    float s[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
        s[c] = ((x.m[c][0] * y.m[c][0] + x.m[c][1] * y.m[c][1]) + x.m[c][2] * y.m[c][2]) + x.m[c][3] * y.m[c][3];
    return ((s[0] + s[1]) + s[2]) + s[3];
}

// Inverse through the adjugate: 2x2 minors of the first two and last two
// columns, then cofactors scaled by 1/det.
__host__ __device__ inline M4 m4_inverse(const M4& a) {
    const float (*m)[4] = a.m;
    const float s0 = m[0][0] * m[1][1] - m[1][0] * m[0][1];
    const float s1 = m[0][0] * m[1][2] - m[1][0] * m[0][2];
    const float s2 = m[0][0] * m[1][3] - m[1][0] * m[0][3];
    const float s3 = m[0][1] * m[1][2] - m[1][1] * m[0][2];
    const float s4 = m[0][1] * m[1][3] - m[1][1] * m[0][3];
    const float s5 = m[0][2] * m[1][3] - m[1][2] * m[0][3];
    const float c5 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
    const float c4 = m[2][1] * m[3][3] - m[3][1] * m[2][3];
    const float c3 = m[2][1] * m[3][2] - m[3][1] * m[2][2];
    const float c2 = m[2][0] * m[3][3] - m[3][0] * m[2][3];
    const float c1 = m[2][0] * m[3][2] - m[3][0] * m[2][2];
    const float c0 = m[2][0] * m[3][1] - m[3][0] * m[2][1];
    const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    const float id = 1.0f / det;
    M4 r;
    r.m[0][0] = (m[1][1] * c5 - m[1][2] * c4 + m[1][3] * c3) * id;
    r.m[0][1] = (-m[0][1] * c5 + m[0][2] * c4 - m[0][3] * c3) * id;
    r.m[0][2] = (m[3][1] * s5 - m[3][2] * s4 + m[3][3] * s3) * id;
    r.m[0][3] = (-m[2][1] * s5 + m[2][2] * s4 - m[2][3] * s3) * id;
    r.m[1][0] = (-m[1][0] * c5 + m[1][2] * c2 - m[1][3] * c1) * id;
    r.m[1][1] = (m[0][0] * c5 - m[0][2] * c2 + m[0][3] * c1) * id;
    r.m[1][2] = (-m[3][0] * s5 + m[3][2] * s2 - m[3][3] * s1) * id;
    r.m[1][3] = (m[2][0] * s5 - m[2][2] * s2 + m[2][3] * s1) * id;
    r.m[2][0] = (m[1][0] * c4 - m[1][1] * c2 + m[1][3] * c0) * id;
    r.m[2][1] = (-m[0][0] * c4 + m[0][1] * c2 - m[0][3] * c0) * id;
    r.m[2][2] = (m[3][0] * s4 - m[3][1] * s2 + m[3][3] * s0) * id;
    r.m[2][3] = (-m[2][0] * s4 + m[2][1] * s2 - m[2][3] * s0) * id;
    r.m[3][0] = (-m[1][0] * c3 + m[1][1] * c1 - m[1][2] * c0) * id;
    r.m[3][1] = (m[0][0] * c3 - m[0][1] * c1 + m[0][2] * c0) * id;
    r.m[3][2] = (-m[3][0] * s3 + m[3][1] * s1 - m[3][2] * s0) * id;
    r.m[3][3] = (m[2][0] * s3 - m[2][1] * s1 + m[2][2] * s0) * id;
    return r;
}

}  // namespace arp
