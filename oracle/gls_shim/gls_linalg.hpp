// gls_linalg.hpp — TEST INFRASTRUCTURE ONLY. A stand-in for the fixed-size
// Vector / Matrix types of the un-vendored GlassImage library, restricted to
// what the reference's ImageRegistration sources use (SURF.cpp,
// LeastSquaresHomography.cpp, Homography.cpp/.hpp).
//
// Arithmetic is one IEEE operation per element, in this order:
//   * Matrix * Matrix: out[i][j] = sum over k = 0.. of a[i][k] * b[k][j],
//     accumulated left to right from 0;
//   * dot(a, b): sum over i = 0.. of a[i] * b[i], left to right from 0;
//   * element-wise + - / and division by a scalar divide each element;
//   * inverse of a 3x3: adjugate divided by the determinant.
// The registration oracle (oracle/gls_oracle_reg.hpp) assumes the same
// reading of these operations.
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <initializer_list>

#include "gls_image.hpp"

namespace gls {

template <size_t N, class T = float>
struct Vector : std::array<T, N> {
    Vector() : std::array<T, N>{} {}
    Vector(std::initializer_list<T> v) : std::array<T, N>{} {
        size_t i = 0;
        for (const T& x : v) (*this)[i++] = x;
    }
    template <class U>
    explicit Vector(const basic_point<U>& p) : std::array<T, N>{} {
        static_assert(N == 2, "a point is a 2-vector");
        (*this)[0] = T(p.x);
        (*this)[1] = T(p.y);
    }
    static Vector zeros() { return Vector(); }

    Vector& operator+=(const Vector& o) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] + o[i];
        return *this;
    }
    Vector& operator-=(const Vector& o) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] - o[i];
        return *this;
    }
    Vector& operator/=(T s) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] / s;
        return *this;
    }
};

template <size_t N, class T>
Vector<N, T> operator+(Vector<N, T> a, const Vector<N, T>& b) {
    return a += b;
}
template <size_t N, class T>
Vector<N, T> operator-(Vector<N, T> a, const Vector<N, T>& b) {
    return a -= b;
}
template <size_t N, class T>
Vector<N, T> operator/(Vector<N, T> a, const Vector<N, T>& b) {
    for (size_t i = 0; i < N; i++) a[i] = a[i] / b[i];
    return a;
}
template <size_t N, class T>
Vector<N, T> operator/(Vector<N, T> a, T s) {
    return a /= s;
}
template <size_t N, class T>
Vector<N, T> abs(Vector<N, T> a) {
    for (size_t i = 0; i < N; i++) a[i] = std::abs(a[i]);
    return a;
}
template <size_t N, class T>
T dot(const Vector<N, T>& a, const Vector<N, T>& b) {
    T s = 0;
    for (size_t i = 0; i < N; i++) s = s + a[i] * b[i];
    return s;
}

template <size_t N, size_t M, class T = float>
struct Matrix : std::array<Vector<M, T>, N> {
    Matrix() : std::array<Vector<M, T>, N>{} {}
    Matrix(std::initializer_list<T> flat) : std::array<Vector<M, T>, N>{} {  // row-major
        size_t k = 0;
        for (const T& x : flat) {
            (*this)[k / M][k % M] = x;
            k++;
        }
    }
    Matrix(std::initializer_list<Vector<M, T>> rows) : std::array<Vector<M, T>, N>{} {
        size_t i = 0;
        for (const auto& r : rows) (*this)[i++] = r;
    }
    template <class U>
    explicit Matrix(const Vector<N * M, U>& v) : std::array<Vector<M, T>, N>{} {  // row-major
        for (size_t k = 0; k < N * M; k++) (*this)[k / M][k % M] = T(v[k]);
    }
    template <class U>
    explicit Matrix(const Matrix<N, M, U>& o) : std::array<Vector<M, T>, N>{} {
        for (size_t i = 0; i < N; i++)
            for (size_t j = 0; j < M; j++) (*this)[i][j] = T(o[i][j]);
    }
    static Matrix zeros() { return Matrix(); }
    static Matrix identity() {
        Matrix r;
        for (size_t i = 0; i < N && i < M; i++) r[i][i] = 1;
        return r;
    }
};

template <size_t N, size_t K, size_t M, class T>
Matrix<N, M, T> operator*(const Matrix<N, K, T>& a, const Matrix<K, M, T>& b) {
    Matrix<N, M, T> r;
    for (size_t i = 0; i < N; i++)
        for (size_t j = 0; j < M; j++) {
            T s = 0;
            for (size_t k = 0; k < K; k++) s = s + a[i][k] * b[k][j];
            r[i][j] = s;
        }
    return r;
}
template <size_t N, size_t M, class T>
Matrix<N, M, T> operator/(Matrix<N, M, T> a, T s) {
    for (size_t i = 0; i < N; i++)
        for (size_t j = 0; j < M; j++) a[i][j] = a[i][j] / s;
    return a;
}
template <class T>
Matrix<3, 3, T> inverse(const Matrix<3, 3, T>& m) {
    const T c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    const T c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    const T c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    const T det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    Matrix<3, 3, T> r = {c00,
                         m[0][2] * m[2][1] - m[0][1] * m[2][2],
                         m[0][1] * m[1][2] - m[0][2] * m[1][1],
                         c01,
                         m[0][0] * m[2][2] - m[0][2] * m[2][0],
                         m[0][2] * m[1][0] - m[0][0] * m[1][2],
                         c02,
                         m[0][1] * m[2][0] - m[0][0] * m[2][1],
                         m[0][0] * m[1][1] - m[0][1] * m[1][0]};
    return r / det;
}

}  // namespace gls
