// gls_image.hpp — TEST INFRASTRUCTURE ONLY. A stand-in for the point, size,
// rectangle and image types of the GlassImage library, which the reference's
// ImageRegistration sources include but the reference tree does not carry
// (an un-vendored submodule). Only what those sources use is defined, so
// that the reference's own registration code compiles as the pin of the
// registration oracle (oracle/Makefile, target ref).
//
// gls::image<T> is a row-major view: width, height and a row stride in
// elements over shared storage. A sub-image (image(base, rectangle)) views
// the base image's storage at the rectangle's origin, so negative indices
// reach the pixels above and to the left, as the reference's 3x3x3
// neighbourhood reads do (SURF.cpp:352-356). Copies are views too. New
// images are zero-filled.
#pragma once

#include <cstddef>
#include <memory>
#include <ostream>
#include <vector>

namespace gls {

template <class T>
struct basic_point {
    T x{}, y{};
    basic_point() = default;
    constexpr basic_point(T x_, T y_) : x(x_), y(y_) {}
    basic_point& operator+=(const basic_point& o) {
        x += o.x;
        y += o.y;
        return *this;
    }
    basic_point& operator-=(const basic_point& o) {
        x -= o.x;
        y -= o.y;
        return *this;
    }
    basic_point& operator*=(T s) {
        x *= s;
        y *= s;
        return *this;
    }
    basic_point& operator/=(T s) {
        x /= s;
        y /= s;
        return *this;
    }
    bool operator==(const basic_point& o) const { return x == o.x && y == o.y; }
};

template <class T>
basic_point<T> operator+(basic_point<T> a, const basic_point<T>& b) {
    return a += b;
}
template <class T>
basic_point<T> operator-(basic_point<T> a, const basic_point<T>& b) {
    return a -= b;
}
template <class T>
std::ostream& operator<<(std::ostream& os, const basic_point<T>& p) {
    return os << "{" << p.x << ", " << p.y << "}";
}

typedef basic_point<int> point;

struct size {
    int width = 0, height = 0;
    bool operator==(const size& o) const { return width == o.width && height == o.height; }
};

struct rectangle {
    int x = 0, y = 0, width = 0, height = 0;
    rectangle() = default;
    constexpr rectangle(int x_, int y_, int w_, int h_) : x(x_), y(y_), width(w_), height(h_) {}
};

template <class T>
class image {
   public:
    typedef std::unique_ptr<image<T>> unique_ptr;

    int width = 0, height = 0, stride = 0;

    image(int w, int h)
        : width(w), height(h), stride(w), _store(std::make_shared<std::vector<T>>(size_t(w) * size_t(h))) {
        _data = _store->data();
    }
    image(const image& base, const rectangle& r)
        : width(r.width), height(r.height), stride(base.stride), _store(base._store),
          _data(base._data + std::ptrdiff_t(r.y) * base.stride + r.x) {}
    image(image* base, const rectangle& r) : image(*base, r) {}
    image(const image&) = default;
    image& operator=(const image&) = default;

    T* operator[](int row) { return _data + std::ptrdiff_t(row) * stride; }
    const T* operator[](int row) const { return _data + std::ptrdiff_t(row) * stride; }
    gls::size size() const { return {width, height}; }
    T* data() { return _data; }

   private:
    std::shared_ptr<std::vector<T>> _store;
    T* _data = nullptr;
};

}  // namespace gls
