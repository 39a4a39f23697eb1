// glsl.hpp -- GLSL 4.60 value semantics for the CPU oracle (test infrastructure).
//
// vec4 / mat4 with GLSL's conventions: mat4 is column-major (m[c][r]),
// `m * v` combines columns, `outerProduct(a, b)` = a b^T, `inverse` is the
// adjugate / determinant form.  Evaluation order of every sum is fixed
// (left to right) so float results are reproducible; the oracle is compiled
// with -ffp-contract=off so no multiply-add is fused behind its back.
#pragma once
#include <cmath>

namespace glsl {

template <class T>
struct vec4 {
    T v[4];
    vec4() : v{0, 0, 0, 0} {}
    vec4(T a, T b, T c, T d) : v{a, b, c, d} {}
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
};

template <class T> inline vec4<T> operator+(const vec4<T>& a, const vec4<T>& b) {
    return {a[0] + b[0], a[1] + b[1], a[2] + b[2], a[3] + b[3]};
}
template <class T> inline vec4<T> operator-(const vec4<T>& a, const vec4<T>& b) {
    return {a[0] - b[0], a[1] - b[1], a[2] - b[2], a[3] - b[3]};
}
template <class T> inline vec4<T> operator-(const vec4<T>& a) { return {-a[0], -a[1], -a[2], -a[3]}; }
template <class T> inline vec4<T> operator*(T s, const vec4<T>& a) {
    return {s * a[0], s * a[1], s * a[2], s * a[3]};
}
template <class T> inline vec4<T> operator*(const vec4<T>& a, T s) {
    return {a[0] * s, a[1] * s, a[2] * s, a[3] * s};
}
template <class T> inline vec4<T> operator/(const vec4<T>& a, T s) {
    return {a[0] / s, a[1] / s, a[2] / s, a[3] / s};
}
template <class T> inline vec4<T>& operator+=(vec4<T>& a, const vec4<T>& b) { a = a + b; return a; }
template <class T> inline vec4<T>& operator-=(vec4<T>& a, const vec4<T>& b) { a = a - b; return a; }

template <class T> inline T dot(const vec4<T>& a, const vec4<T>& b) {
    return ((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]) + a[3] * b[3];
}
template <class T> inline T length(const vec4<T>& a) { return std::sqrt(dot(a, a)); }
template <class T> inline vec4<T> normalize(const vec4<T>& a) { return a / length(a); }
template <class T> inline bool any_nan_or_inf(const vec4<T>& a) {
    for (int i = 0; i < 4; ++i)
        if (std::isnan(a[i]) || std::isinf(a[i])) return true;
    return false;
}

template <class T>
struct mat4 {
    vec4<T> c[4];  // columns
    mat4() {}
    explicit mat4(T d) {
        for (int i = 0; i < 4; ++i) c[i][i] = d;
    }
    vec4<T>& operator[](int i) { return c[i]; }
    const vec4<T>& operator[](int i) const { return c[i]; }
};

template <class T> inline mat4<T> identity() { return mat4<T>(T(1)); }

template <class T> inline mat4<T> operator+(const mat4<T>& a, const mat4<T>& b) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i) r[i] = a[i] + b[i];
    return r;
}
template <class T> inline mat4<T> operator-(const mat4<T>& a, const mat4<T>& b) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i) r[i] = a[i] - b[i];
    return r;
}
template <class T> inline mat4<T> operator-(const mat4<T>& a) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i) r[i] = -a[i];
    return r;
}
template <class T> inline mat4<T> operator*(T s, const mat4<T>& a) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i) r[i] = s * a[i];
    return r;
}
template <class T> inline mat4<T> operator/(const mat4<T>& a, T s) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i) r[i] = a[i] / s;
    return r;
}
// m * v = sum over columns c of m[c] * v[c]
template <class T> inline vec4<T> operator*(const mat4<T>& m, const vec4<T>& v) {
    vec4<T> r;
    for (int row = 0; row < 4; ++row)
        r[row] = ((m[0][row] * v[0] + m[1][row] * v[1]) + m[2][row] * v[2]) + m[3][row] * v[3];
    return r;
}
template <class T> inline mat4<T> operator*(const mat4<T>& a, const mat4<T>& b) {
    mat4<T> r;
    for (int col = 0; col < 4; ++col) r[col] = a * b[col];
    return r;
}
template <class T> inline mat4<T>& operator+=(mat4<T>& a, const mat4<T>& b) { a = a + b; return a; }
template <class T> inline mat4<T>& operator*=(mat4<T>& a, const mat4<T>& b) { a = a * b; return a; }

template <class T> inline mat4<T> transpose(const mat4<T>& a) {
    mat4<T> r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) r[i][j] = a[j][i];
    return r;
}
// outerProduct(c, r): column vector c times row vector r; result[col][row] = c[row] * r[col]
template <class T> inline mat4<T> outerProduct(const vec4<T>& c, const vec4<T>& r) {
    mat4<T> m;
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) m[col][row] = c[row] * r[col];
    return m;
}

// 4x4 inverse by cofactor expansion along 2x2 sub-determinants.
template <class T> inline mat4<T> inverse(const mat4<T>& m) {
    const T a00 = m[0][0], a01 = m[0][1], a02 = m[0][2], a03 = m[0][3];
    const T a10 = m[1][0], a11 = m[1][1], a12 = m[1][2], a13 = m[1][3];
    const T a20 = m[2][0], a21 = m[2][1], a22 = m[2][2], a23 = m[2][3];
    const T a30 = m[3][0], a31 = m[3][1], a32 = m[3][2], a33 = m[3][3];
    const T b00 = a00 * a11 - a01 * a10, b01 = a00 * a12 - a02 * a10;
    const T b02 = a00 * a13 - a03 * a10, b03 = a01 * a12 - a02 * a11;
    const T b04 = a01 * a13 - a03 * a11, b05 = a02 * a13 - a03 * a12;
    const T b06 = a20 * a31 - a21 * a30, b07 = a20 * a32 - a22 * a30;
    const T b08 = a20 * a33 - a23 * a30, b09 = a21 * a32 - a22 * a31;
    const T b10 = a21 * a33 - a23 * a31, b11 = a22 * a33 - a23 * a32;
    const T det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06;
    const T inv = T(1) / det;
    mat4<T> r;
    r[0][0] = (a11 * b11 - a12 * b10 + a13 * b09) * inv;
    r[0][1] = (a02 * b10 - a01 * b11 - a03 * b09) * inv;
    r[0][2] = (a31 * b05 - a32 * b04 + a33 * b03) * inv;
    r[0][3] = (a22 * b04 - a21 * b05 - a23 * b03) * inv;
    r[1][0] = (a12 * b08 - a10 * b11 - a13 * b07) * inv;
    r[1][1] = (a00 * b11 - a02 * b08 + a03 * b07) * inv;
    r[1][2] = (a32 * b02 - a30 * b05 - a33 * b01) * inv;
    r[1][3] = (a20 * b05 - a22 * b02 + a23 * b01) * inv;
    r[2][0] = (a10 * b10 - a11 * b08 + a13 * b06) * inv;
    r[2][1] = (a01 * b08 - a00 * b10 - a03 * b06) * inv;
    r[2][2] = (a30 * b04 - a31 * b02 + a33 * b00) * inv;
    r[2][3] = (a21 * b02 - a20 * b04 - a23 * b00) * inv;
    r[3][0] = (a11 * b07 - a10 * b09 - a12 * b06) * inv;
    r[3][1] = (a00 * b09 - a01 * b07 + a02 * b06) * inv;
    r[3][2] = (a31 * b01 - a30 * b03 - a32 * b00) * inv;
    r[3][3] = (a20 * b03 - a21 * b01 + a22 * b00) * inv;
    return r;
}

// x^7 by explicit products, used wherever the shaders call pow(x, 7).
template <class T> inline T pow7(T x) {
    const T x2 = x * x;
    const T x3 = x2 * x;
    const T x6 = x3 * x3;
    return x6 * x;
}

}  // namespace glsl
