// glm/glm.hpp -- minimal host stand-in for the parts of the GLM matrix library that the
// reference's rasterizer uses (TEST INFRASTRUCTURE ONLY; GLM itself is not vendored with
// the reference and no version is pinned).  It restates GLM's published conventions:
//   * mat3 is column-major: m[c] is column c, m[c][r] the element in row r;
//     mat3(s) puts s on the diagonal; mat3(a0..a8) fills column 0 with a0..a2, column 1
//     with a3..a5, column 2 with a6..a8;
//   * (A * B)[c][r] = A[0][r] * B[c][0] + A[1][r] * B[c][1] + A[2][r] * B[c][2], summed left
//     to right, each product and sum rounded to float (the definition of the product);
//   * s * A and A * s scale every element; -A negates every element;
//   * transpose(A)[c][r] = A[r][c]; sign(x) = -1, 0 or 1.
#pragma once

namespace glm {

struct vec3 {
    float x, y, z;
    vec3() : x(0.f), y(0.f), z(0.f) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const float& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec3& operator*=(float s) {
        x *= s;
        y *= s;
        z *= s;
        return *this;
    }
};

struct vec4 {
    float x, y, z, w;
    vec4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};

struct mat3 {
    vec3 c[3];
    mat3() : mat3(1.0f) {}
    explicit mat3(float s) {
        c[0] = vec3(s, 0.f, 0.f);
        c[1] = vec3(0.f, s, 0.f);
        c[2] = vec3(0.f, 0.f, s);
    }
    mat3(float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, float a8) {
        c[0] = vec3(a0, a1, a2);
        c[1] = vec3(a3, a4, a5);
        c[2] = vec3(a6, a7, a8);
    }
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};

inline mat3 operator*(const mat3& A, const mat3& B) {
    mat3 R(0.f);
    for (int col = 0; col < 3; col++)
        for (int row = 0; row < 3; row++) {
            float s = A[0][row] * B[col][0];
            s = s + A[1][row] * B[col][1];
            s = s + A[2][row] * B[col][2];
            R[col][row] = s;
        }
    return R;
}

inline mat3 operator*(float s, const mat3& A) {
    mat3 R(0.f);
    for (int col = 0; col < 3; col++)
        for (int row = 0; row < 3; row++) R[col][row] = s * A[col][row];
    return R;
}

inline mat3 operator*(const mat3& A, float s) {
    mat3 R(0.f);
    for (int col = 0; col < 3; col++)
        for (int row = 0; row < 3; row++) R[col][row] = A[col][row] * s;
    return R;
}

inline mat3 operator-(const mat3& A) {
    mat3 R(0.f);
    for (int col = 0; col < 3; col++)
        for (int row = 0; row < 3; row++) R[col][row] = -A[col][row];
    return R;
}

inline mat3 transpose(const mat3& A) {
    mat3 R(0.f);
    for (int col = 0; col < 3; col++)
        for (int row = 0; row < 3; row++) R[col][row] = A[row][col];
    return R;
}

inline float sign(float x) { return (float)((0.f < x) - (x < 0.f)); }

}  // namespace glm
