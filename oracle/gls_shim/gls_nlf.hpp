// gls_nlf.hpp — TEST INFRASTRUCTURE ONLY. Stand-ins for the GlassImage
// vector and image types (an un-vendored submodule of the reference) with
// what the reference's noise-model regressions use
// (RawConverter::MeasureRawNLF, raw_converter.cpp:339-490, and
// PyramidProcessor::MeasureYCbCrNLF, pyramid_processor.cpp:173-324), so
// that those functions compile unmodified as the pin of the oracle's
// restatement (oracle/ref_nlf.cpp). Used by that translation unit only.
//
// Semantics:
//   * Vector<N, T> is an array with element-wise arithmetic, one IEEE
//     operation per element; a scalar operand applies to every element;
//   * comparisons, isnan and the like are element-wise and give a BVector;
//     any() / all() reduce it; a BVector used as a condition means all()
//     (the reference's `newErr2 < err2` in an && expression,
//     raw_converter.cpp:463; its sibling check reads all(newErr2 <= err2),
//     pyramid_processor.cpp:294);
//   * apply(f, v) maps f over the elements; max_element(v) is the largest
//     element's value;
//   * image<T>::apply(f) calls f(pixel, x, y) row by row, left to right.
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <ostream>
#include <vector>

namespace gls {

template <size_t N>
struct BVector : std::array<bool, N> {
    explicit operator bool() const {
        for (bool b : *this)
            if (!b) return false;
        return true;
    }
};

template <size_t N, class T = float>
struct Vector : std::array<T, N> {
    Vector() : std::array<T, N>{} {}
    Vector(T s) : std::array<T, N>{} {  // a scalar fills every element
        for (auto& e : *this) e = s;
    }
    Vector(std::initializer_list<T> v) : std::array<T, N>{} {
        size_t i = 0;
        for (const T& x : v) (*this)[i++] = x;
    }
    template <class U>
    Vector(const Vector<N, U>& o) : std::array<T, N>{} {
        for (size_t i = 0; i < N; i++) (*this)[i] = T(o[i]);
    }
    Vector& operator+=(const Vector& o) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] + o[i];
        return *this;
    }
    Vector& operator-=(const Vector& o) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] - o[i];
        return *this;
    }
    Vector& operator*=(T s) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] * s;
        return *this;
    }
    Vector& operator/=(T s) {
        for (size_t i = 0; i < N; i++) (*this)[i] = (*this)[i] / s;
        return *this;
    }
};

template <size_t N>
using DVector = Vector<N, double>;

#define GLS_NLF_BINOP(OP)                                                     \
    template <size_t N, class T>                                             \
    Vector<N, T> operator OP(const Vector<N, T>& a, const Vector<N, T>& b) { \
        Vector<N, T> r;                                                      \
        for (size_t i = 0; i < N; i++) r[i] = a[i] OP b[i];                  \
        return r;                                                            \
    }                                                                        \
    template <size_t N, class T>                                             \
    Vector<N, T> operator OP(const Vector<N, T>& a, T s) {                   \
        Vector<N, T> r;                                                      \
        for (size_t i = 0; i < N; i++) r[i] = a[i] OP s;                     \
        return r;                                                            \
    }                                                                        \
    template <size_t N, class T>                                             \
    Vector<N, T> operator OP(T s, const Vector<N, T>& b) {                   \
        Vector<N, T> r;                                                      \
        for (size_t i = 0; i < N; i++) r[i] = s OP b[i];                     \
        return r;                                                            \
    }
GLS_NLF_BINOP(+)
GLS_NLF_BINOP(-)
GLS_NLF_BINOP(*)
GLS_NLF_BINOP(/)
#undef GLS_NLF_BINOP

#define GLS_NLF_CMP(OP)                                                   \
    template <size_t N, class T>                                         \
    BVector<N> operator OP(const Vector<N, T>& a, const Vector<N, T>& b) { \
        BVector<N> r;                                                    \
        for (size_t i = 0; i < N; i++) r[i] = a[i] OP b[i];              \
        return r;                                                        \
    }
GLS_NLF_CMP(<)
GLS_NLF_CMP(<=)
GLS_NLF_CMP(>)
GLS_NLF_CMP(>=)
#undef GLS_NLF_CMP

template <size_t N>
bool any(const BVector<N>& v) {
    for (bool b : v)
        if (b) return true;
    return false;
}
template <size_t N>
bool all(const BVector<N>& v) {
    for (bool b : v)
        if (!b) return false;
    return true;
}
template <size_t N, class T>
BVector<N> isnan(const Vector<N, T>& v) {
    BVector<N> r;
    for (size_t i = 0; i < N; i++) r[i] = std::isnan(v[i]);
    return r;
}
template <size_t N, class T>
Vector<N, T> abs(const Vector<N, T>& v) {
    Vector<N, T> r;
    for (size_t i = 0; i < N; i++) r[i] = std::abs(v[i]);
    return r;
}
template <size_t N, class T>
Vector<N, T> sqrt(const Vector<N, T>& v) {
    Vector<N, T> r;
    for (size_t i = 0; i < N; i++) r[i] = std::sqrt(v[i]);
    return r;
}
template <size_t N, class T>
Vector<N, T> max(const Vector<N, T>& v, T s) {
    Vector<N, T> r;
    for (size_t i = 0; i < N; i++) r[i] = v[i] > s ? v[i] : s;
    return r;
}
template <size_t N, class T>
T max_element(const Vector<N, T>& v) {
    T m = v[0];
    for (size_t i = 1; i < N; i++)
        if (v[i] > m) m = v[i];
    return m;
}
template <size_t N>
Vector<N, double> apply(double (*f)(double), const Vector<N, double>& v) {
    Vector<N, double> r;
    for (size_t i = 0; i < N; i++) r[i] = f(v[i]);
    return r;
}
template <size_t N, class T>
std::ostream& operator<<(std::ostream& os, const Vector<N, T>& v) {
    os << "{";
    for (size_t i = 0; i < N; i++) os << (i ? ", " : "") << v[i];
    return os << "}";
}

struct size {
    int width = 0, height = 0;
    bool operator==(const size& o) const { return width == o.width && height == o.height; }
};

// an RGBA float pixel: .v the 4-vector, [i] its elements
struct pixel_float4 {
    Vector<4, float> v;
    float operator[](int i) const { return v[size_t(i)]; }
};
typedef float pixel_float;
typedef uint16_t luma_pixel_16;

template <class T>
struct image {
    int width = 0, height = 0;
    std::vector<T> px;
    image(int w, int h) : width(w), height(h), px(size_t(w) * size_t(h)) {}
    T* operator[](int row) { return px.data() + size_t(row) * width; }
    const T* operator[](int row) const { return px.data() + size_t(row) * width; }
    gls::size size() const { return {width, height}; }
    template <class F>
    void apply(F f) const {
        for (int y = 0; y < height; y++)
            for (int x = 0; x < width; x++) f((*this)[y][x], x, y);
    }
};

// the Metal texture of the reference: here host memory, mapped in place
template <class T>
struct mtl_image_2d : image<T> {
    using image<T>::image;
    const image<T>* mapImage() const { return this; }
};

}  // namespace gls
