// gls_oracle.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the
// GlassCamera raw path (demosaic, high-noise raw denoise, pyramid PCA
// block-matching denoise and reconstruct) used as the checker for the CUDA
// library. Nothing in the product links or calls this code; only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
//
// Every function cites the reference file:line it restates (paths relative
// to the GlassCameraPublic tree). The arithmetic is templated on the scalar
// type T: T = double is the "truth" run, T = float the FP32 run. Parameters
// that the reference computes on the host in float (tap weights, colour
// matrices, noise model) are float in both modes.
//
// Semantics the reference leaves undefined, fixed here and in the CUDA
// kernels alike:
//   * texture reads outside the image clamp to the edge (Metal leaves
//     out-of-bounds read() undefined);
//   * sampler(filter::linear) is exact bilinear interpolation at texel-space
//     position (normalised coordinate * size - 0.5), clamp-to-edge;
//   * the PCA patch sample set is the (W/8) x (H/8) grid of patches, packed
//     densely (the reference's y*width/8 + x indexing leaves stale entries
//     in its sample span, demosaic.metal:768, pyramid_processor.cpp:141-149).
//
// Parity of this restatement against the reference: the reference cannot be
// built or run here (Metal kernels, Apple frameworks, un-vendored GlassImage
// submodule, Eigen), and it ships no tests or golden vectors. Where the
// Metal kernel source itself compiles as C++ under oracle/metal_shim (see
// oracle/Makefile), tests compare this restatement with it; elsewhere parity
// rests on the known-answer tests under tests/.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- threading
inline int& num_threads() {
    static int n = std::max(1u, std::thread::hardware_concurrency());
    return n;
}

template <class F>
void parallel_rows(int rows, F&& fn) {
    const int nt = std::max(1, std::min(num_threads(), rows));
    if (nt == 1) {
        for (int y = 0; y < rows; y++) fn(y);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int t = 0; t < nt; t++) {
        th.emplace_back([&, t]() {
            for (int y = t; y < rows; y += nt) fn(y);
        });
    }
    for (auto& x : th) x.join();
}

// ---------------------------------------------------------------- images
// Interleaved C-channel image with clamp-to-edge reads.
template <class T, int C>
struct Img {
    int w = 0, h = 0;
    std::vector<T> d;
    Img() = default;
    Img(int w_, int h_) : w(w_), h(h_), d(size_t(w_) * h_ * C, T(0)) {}
    T* px(int x, int y) { return &d[(size_t(y) * w + x) * C]; }
    const T* px(int x, int y) const { return &d[(size_t(y) * w + x) * C]; }
    // clamp-to-edge read of channel c
    T at(int x, int y, int c = 0) const {
        x = std::clamp(x, 0, w - 1);
        y = std::clamp(y, 0, h - 1);
        return d[(size_t(y) * w + x) * C + c];
    }
    // bilinear sample at texel (xi + fx, yi + fy), fx, fy in [0, 1),
    // clamp-to-edge; the integer and fractional parts stay separate so the
    // position is exact at any image size
    T bilin_split(int xi, T ax, int yi, T ay, int c) const {
        const T a = at(xi, yi, c), b = at(xi + 1, yi, c);
        const T cc = at(xi, yi + 1, c), dd = at(xi + 1, yi + 1, c);
        const T top = a + (b - a) * ax;
        const T bot = cc + (dd - cc) * ax;
        return top + (bot - top) * ay;
    }
    // bilinear sample at texel-space position (u, v), clamp-to-edge
    T bilin(T u, T v, int c) const {
        const T fu = std::floor(u), fv = std::floor(v);
        const int x0 = int(fu), y0 = int(fv);
        const T ax = u - fu, ay = v - fv;
        const T a = at(x0, y0, c), b = at(x0 + 1, y0, c);
        const T cc = at(x0, y0 + 1, c), dd = at(x0 + 1, y0 + 1, c);
        const T top = a + (b - a) * ax;
        const T bot = cc + (dd - cc) * ax;
        return top + (bot - top) * ay;
    }
};

// ---------------------------------------------------------------- math
template <class T>
inline T clampT(T x, T lo, T hi) {  // Metal clamp = min(max(x, lo), hi)
    return std::min(std::max(x, lo), hi);
}
template <class T>
inline T smoothstepT(T e0, T e1, T x) {
    T t = clampT<T>((x - e0) / (e1 - e0), T(0), T(1));
    return t * t * (T(3) - T(2) * t);
}
template <class T>
inline T mixT(T a, T b, T t) {
    return a + (b - a) * t;
}
// gaussian(x) = exp(-2 x^2), demosaic.metal:87-89
template <class T>
inline T gaussianT(T x) {
    return std::exp(T(-2) * x * x);
}
template <class T>
inline T pi_v() {
    return T(3.14159265358979323846);
}

// Bayer channel offsets (x, y) of R, G, B, G2 inside a 2x2 quad, in the
// order the Metal kernels use them (demosaic.metal:33-38). The host-side
// table in demosaic.hpp:128-133 swaps G and G2; the kernels' table wins.
static const int kBayerOffsets[4][4][2] = {
    {{1, 0}, {0, 0}, {0, 1}, {1, 1}},  // grbg
    {{0, 1}, {0, 0}, {1, 0}, {1, 1}},  // gbrg
    {{0, 0}, {0, 1}, {1, 1}, {1, 0}},  // rggb
    {{1, 1}, {0, 1}, {0, 0}, {1, 0}},  // bggr
};

// Bayer channel (0=R, 1=G, 2=B, 3=G2) of pixel (x, y).
inline int bayer_channel(int pattern, int x, int y) {
    for (int c = 0; c < 4; c++) {
        if (kBayerOffsets[pattern][c][0] == (x & 1) && kBayerOffsets[pattern][c][1] == (y & 1)) return c;
    }
    return 0;
}

// ---------------------------------------------------------------- params
struct Taps {
    std::vector<std::array<float, 3>> t;  // (weight, dx, dy)
};

// gaussianKernelBilinearWeights + KernelOptimizeBilinear2d,
// demosaic_utils.cpp:934-1006. A (2k+1)^2 Gaussian is folded into
// (k+1)^2 bilinear taps. The last tap's offsets are width/2.0f, as the
// reference writes them (demosaic_utils.cpp:984), not width/2.
inline Taps gaussian_bilinear_taps(float radius) {
    int ks = std::max(int(std::ceil(2 * radius)), 2);
    if ((ks % 2) == 0) ks++;
    std::vector<float> w(size_t(ks) * ks);
    for (int y = -ks / 2, i = 0; y <= ks / 2; y++)
        for (int x = -ks / 2; x <= ks / 2; x++, i++)
            w[i] = float(std::exp(-(double(float(x * x + y * y)) / double(2 * radius * radius))));
    const int ow = ks / 2 + 1, half = ks / 2;
    Taps out;
    out.t.assign(size_t(ow) * ow, {0, 0, 0});
    int row, col;
    for (row = 0; row < ks - 1; row += 2) {
        for (col = 0; col < ks - 1; col += 2) {
            float w1 = w[row * ks + col], w2 = w[row * ks + col + 1];
            float w3 = w[(row + 1) * ks + col], w4 = w[(row + 1) * ks + col + 1];
            float x1 = float(col - half), x2 = float(col - half + 1);
            float y1 = float(row - half), y2 = float(row - half + 1);
            out.t[(row / 2) * ow + col / 2] = {w1 + w2 + w3 + w4, (x1 * w1 + x2 * w2) / (w1 + w2),
                                               (y1 * w1 + y2 * w3) / (w1 + w3)};
        }
        float w1 = w[row * ks + col], w2 = w[(row + 1) * ks + col];
        float y1 = float(row - half), y2 = float(row - half + 1);
        out.t[(row / 2) * ow + col / 2] = {w1 + w2, float(col - half), (y1 * w1 + y2 * w2) / (w1 + w2)};
    }
    for (col = 0; col < ks - 1; col += 2) {
        float w1 = w[row * ks + col], w2 = w[row * ks + col + 1];
        float x1 = float(col - half), x2 = float(col - half + 1);
        out.t[(row / 2) * ow + col / 2] = {w1 + w2, (x1 * w1 + x2 * w2) / (w1 + w2), float(row - half)};
    }
    out.t[(row / 2) * ow + col / 2] = {w[row * ks + col], ks / 2.0f, ks / 2.0f};
    return out;
}

struct Mat3 {
    float m[3][3];
};

// cam_ycbcr, demosaic_utils.cpp:703-720 (float arithmetic, as the reference).
inline Mat3 cam_ycbcr(const float rgb_cam[9], const float xyz_rgb[9]) {
    float cam_y[3];
    for (int j = 0; j < 3; j++) {
        cam_y[j] = xyz_rgb[3 + 0] * rgb_cam[0 * 3 + j] + xyz_rgb[3 + 1] * rgb_cam[1 * 3 + j] +
                   xyz_rgb[3 + 2] * rgb_cam[2 * 3 + j];
    }
    const float KR = cam_y[0], KG = cam_y[1], KB = cam_y[2];
    Mat3 r = {{{KR, KG, KB},
               {-0.5f * KR / (1.0f - KB), -0.5f * KG / (1 - KB), 0.5f},
               {0.5f, -0.5f * KG / (1 - KR), -0.5f * KB / (1 - KR)}}};
    return r;
}

// 3x3 inverse (raw_converter.cpp:169 calls gls::inverse), computed in
// double and rounded to float.
inline Mat3 inverse3(const Mat3& a) {
    double m[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m[i][j] = a.m[i][j];
    double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    double c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    double c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    double inv[3][3] = {
        {c00, m[0][2] * m[2][1] - m[0][1] * m[2][2], m[0][1] * m[1][2] - m[0][2] * m[1][1]},
        {c01, m[0][0] * m[2][2] - m[0][2] * m[2][0], m[0][2] * m[1][0] - m[0][0] * m[1][2]},
        {c02, m[0][1] * m[2][0] - m[0][0] * m[2][1], m[0][0] * m[1][1] - m[0][1] * m[1][0]}};
    Mat3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = float(inv[i][j] / det);
    return r;
}

struct DenoiseParams {
    float luma = 1, chroma = 1, chromaBoost = 1, gradientBoost = 0, gradientThreshold = 1, sharpening = 1;
};
struct YCbCrNLF {
    float a[3], b[3];
};
struct RawNLF {
    float a[4], b[4];
};

struct Params {
    int bayer = 2;
    float black = 0, white = 65535;
    float lsc = 0;
    float scale_mul[4] = {1, 1, 1, 1};
    float rgb_cam[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float xyz_rgb[9] = {0.4124f, 0.3576f, 0.1805f, 0.2126f, 0.7152f, 0.0722f, 0.0193f, 0.1192f, 0.9505f};
    bool high_noise = false;
    float raw_strength = 1;
    RawNLF raw_nlf{};
    YCbCrNLF pyr_nlf[5]{};
    DenoiseParams dn[5];
    int levels = 5;
};

// getRawVariance, demosaic.hpp:186-193: (red, green, blue) -> (a, b)
inline std::array<std::array<float, 2>, 3> raw_variance(const RawNLF& n) {
    return {{{n.a[0], n.b[0]}, {(n.a[1] + n.a[3]) / 2, (n.b[1] + n.b[3]) / 2}, {n.a[2], n.b[2]}}};
}

// ---------------------------------------------------------------- stages
template <class T>
using Plane = Img<T, 1>;
template <class T>
using Plane2 = Img<T, 2>;
template <class T>
using Plane4 = Img<T, 4>;

// scaleRawData, demosaic.metal:96-118 (grid W/2 x H/2, one quad per thread).
// value = max(ls * scale_mul[c] * (raw - black)/65535 * 0.9 + 0.1, 0).
// The black-level subtraction is exact integer arithmetic here; the factor
// k_c = scale_mul[c] * 0.9 / 65535 is formed in double and rounded to T.
template <class T>
Plane<T> scale_raw(const uint16_t* raw, size_t stride_elems, int w, int h, const Params& p) {
    Plane<T> out(w, h);
    T k[4];
    for (int c = 0; c < 4; c++) k[c] = T(double(p.scale_mul[c]) * 0.9 / 65535.0);
    const int black = int(std::lround(p.black));
    const T cx = T(w / 2), cy = T(h / 2);
    const T clen = std::sqrt(cx * cx + cy * cy);
    parallel_rows(h, [&](int y) {
        for (int x = 0; x < w; x++) {
            T ls = T(1);
            if (p.lsc > 0) {
                // lens shading is evaluated at the quad origin (2 * index)
                const T dx = T(x & ~1) - cx, dy = T(y & ~1) - cy;
                const T r = std::sqrt(dx * dx + dy * dy) / clen;
                ls = T(1) + T(p.lsc) * r * r;
            }
            const int c = bayer_channel(p.bayer, x, y);
            const int d = int(raw[size_t(y) * stride_elems + x]) - black;
            T v = (p.lsc > 0) ? ls * k[c] * T(d) + T(0.1) : T(d) * k[c] + T(0.1);
            out.px(x, y)[0] = std::max(v, T(0));
        }
    });
    return out;
}

// rawImageSobel, demosaic.metal:120-139: (gx, gy, |gx|, |gy|) / sqrt(4.5)
// with gx = left - right and gy = up - down (1-2-1 weights).
template <class T>
Plane4<T> sobel(const Plane<T>& in) {
    Plane4<T> out(in.w, in.h);
    const T inv = T(1) / std::sqrt(T(4.5));
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++) {
            auto r = [&](int i, int j) { return in.at(x + i, y + j); };
            T gx = (r(-1, -1) - r(1, -1)) + T(2) * (r(-1, 0) - r(1, 0)) + (r(-1, 1) - r(1, 1));
            T gy = (r(-1, -1) - r(-1, 1)) + T(2) * (r(0, -1) - r(0, 1)) + (r(1, -1) - r(1, 1));
            gx *= inv;
            gy *= inv;
            T* o = out.px(x, y);
            o[0] = gx;
            o[1] = gy;
            o[2] = std::abs(gx);
            o[3] = std::abs(gy);
        }
    });
    return out;
}

// sampledConvolution over 4 channels, demosaic.metal:175-191; the sample
// point of tap (w, dx, dy) is texel (x + dx, y + dy).
template <class T>
inline void sampled_conv4(const Plane4<T>& s, int x, int y, const Taps& taps, T out[4]) {
    T sum[4] = {0, 0, 0, 0};
    T norm = 0;
    for (const auto& t : taps.t) {
        const T w = T(t[0]);
        const float fdx = std::floor(t[1]), fdy = std::floor(t[2]);
        const int ix = x + int(fdx), iy = y + int(fdy);
        const T ax = T(t[1] - fdx), ay = T(t[2] - fdy);
        for (int c = 0; c < 4; c++) sum[c] += w * s.bilin_split(ix, ax, iy, ay, c);
        norm += w;
    }
    for (int c = 0; c < 4; c++) out[c] = sum[c] / norm;
}

// sampledConvolutionSobel, demosaic.metal:193-213: narrow blur (r=1.5)
// unless |blur(g)| < 4 sigma_raw, then wide blur (r=4.5); output the blurred
// magnitudes with the blurred signs.
template <class T>
Plane2<T> gradient_blur(const Plane<T>& raw, const Plane4<T>& sob, const Taps& t1, const Taps& t2,
                        std::array<float, 2> var) {
    Plane2<T> out(raw.w, raw.h);
    parallel_rows(raw.h, [&](int y) {
        for (int x = 0; x < raw.w; x++) {
            T r[4];
            sampled_conv4(sob, x, y, t1, r);
            const T sigma = std::sqrt(T(var[0]) + T(var[1]) * raw.at(x, y));
            if (std::sqrt(r[0] * r[0] + r[1] * r[1]) < T(4) * sigma) sampled_conv4(sob, x, y, t2, r);
            T* o = out.px(x, y);
            o[0] = std::copysign(r[2], r[0]);
            o[1] = std::copysign(r[3], r[1]);
        }
    });
    return out;
}

// interpolateGreen, demosaic.metal:215-316.
template <class T>
Plane<T> interpolate_green(const Plane<T>& raw, const Plane2<T>& grad, int pattern, std::array<float, 2> gv) {
    Plane<T> out(raw.w, raw.h);
    const int rx = kBayerOffsets[pattern][0][0], ry = kBayerOffsets[pattern][0][1];
    const int bx = kBayerOffsets[pattern][2][0], by = kBayerOffsets[pattern][2][1];
    const T lowNoise = T(1) - smoothstepT<T>(T(3.5e-4f), T(2e-3f), T(gv[1]));
    parallel_rows(raw.h, [&](int y) {
        for (int x = 0; x < raw.w; x++) {
            const bool red = (rx & 1) == (x & 1) && (ry & 1) == (y & 1);
            const bool blue = (bx & 1) == (x & 1) && (by & 1) == (y & 1);
            auto R = [&](int i, int j) { return raw.at(x + i, y + j); };
            if (!(red || blue)) {
                out.px(x, y)[0] = R(0, 0);
                continue;
            }
            const T gl = R(-1, 0), gr = R(1, 0), gu = R(0, -1), gd = R(0, 1);
            const T cxy = R(0, 0);
            const T cl = R(-2, 0), cr = R(2, 0), cu = R(0, -2), cd = R(0, 2);
            const T c2ave = (R(-1, -1) + R(1, -1) + R(-1, 1) + R(1, 1)) / T(4);
            const T gave = (gl + gr + gu + gd) / T(4);
            const T gx = std::abs(grad.at(x, y, 0)), gy = std::abs(grad.at(x, y, 1));
            const T glf_x = (gl + gr) / T(2), glf_y = (gu + gd) / T(2);
            const T ghf_x = ((cl + cr) - T(2) * cxy) / T(4), ghf_y = ((cu + cd) - T(2) * cxy) / T(4);
            const T sd = std::sqrt(T(gv[0]) + T(gv[1]) * gave);
            const T glen = std::sqrt(gx * gx + gy * gy);
            const T gthr = smoothstepT<T>(sd, T(4) * sd, glen);
            const T lowthr = T(1) - smoothstepT<T>(T(2) * sd, T(8) * sd, glen);
            const T sharp = (T(0.5) + T(0.5) * lowNoise) * gthr * (T(1) + lowNoise * lowthr);
            const T hl = T(1) - smoothstepT<T>(T(0.25), T(1), std::max(cxy, std::max(std::max(cl, cr), std::max(cu, cd))));
            T dir = T(2) * std::atan2(gy, gx) / pi_v<T>();
            if (gv[1] < 1e-3f) {
                dir = dir < T(0.5) ? mixT<T>(dir, T(0), T(1) - smoothstepT<T>(T(0.3), T(0.45), dir))
                                   : mixT<T>(dir, T(1), smoothstepT<T>(T(1) - T(0.45), T(1) - T(0.3), dir));
            }
            const T cmin = std::min(cxy, std::min(gave, c2ave));
            const T cmax = std::max(cxy, std::max(gave, c2ave));
            const T white = cmin / cmax;
            const T k = hl * white * sharp;
            const T ge_x = glf_x - k * ghf_x, ge_y = glf_y - k * ghf_y;
            T g = mixT<T>(ge_y, ge_x, dir);
            const T maxo = mixT<T>(T(1), T(1.5), white), mino = mixT<T>(T(1), T(0.5), white);
            const T gmax = std::max(std::max(gl, gr), std::max(gu, gd));
            const T gmin = std::min(std::min(gl, gr), std::min(gu, gd));
            out.px(x, y)[0] = clampT<T>(g, mino * gmin, maxo * gmax);
        }
    });
    return out;
}

// interpolateRedBluePixel, demosaic.metal:327-391 (one R or B site).
template <class T>
inline void rb_at_rb(const Plane<T>& raw, const Plane<T>& green, const Plane2<T>& grad, std::array<float, 2> rv,
                     std::array<float, 2> bv, bool red, int x, int y, T out[3]) {
    auto R = [&](int i, int j) { return raw.at(x + i, y + j); };
    auto G = [&](int i, int j) { return green.at(x + i, y + j); };
    const T g0 = G(0, 0), c1 = R(0, 0);
    const T c2tl = R(-1, -1), c2tr = R(1, -1), c2bl = R(-1, 1), c2br = R(1, 1);
    const T c2ave = (c2tl + c2tr + c2bl + c2br) / T(4);
    const T gctl = G(-1, -1) - c2tl, gctr = G(1, -1) - c2tr, gcbl = G(-1, 1) - c2bl, gcbr = G(1, 1) - c2br;
    const T gtl2 = G(-2, -2), gtr2 = G(2, -2), gbl2 = G(-2, 2), gbr2 = G(2, 2);
    const T gctl2 = gtl2 - R(-2, -2), gctr2 = gtr2 - R(2, -2), gcbl2 = gbl2 - R(-2, 2), gcbr2 = gbr2 - R(2, 2);
    const auto& v = red ? rv : bv;
    const T sd = std::sqrt(T(v[0]) + T(v[1]) * c2ave);
    const T gx = std::abs(grad.at(x, y, 0)), gy = std::abs(grad.at(x, y, 1));
    const T dir = T(1) - T(2) * std::atan2(gy, gx) / pi_v<T>();
    const T gthr = smoothstepT<T>(sd, T(4) * sd, std::sqrt(gx * gx + gy * gy));
    const T alpha = mixT<T>(T(0.5), dir, gthr);
    const T hl = T(1) - smoothstepT<T>(T(0.25), T(1), std::max(g0, std::max(std::max(gtr2, gbl2), std::max(gtl2, gbr2))));
    const T gc = g0 - c1;
    const T a = (gctr + gcbl) / T(2) + hl * (gctr2 + gcbl2 - T(2) * gc) / T(8);
    const T b = (gctl + gcbr) / T(2) + hl * (gctl2 + gcbr2 - T(2) * gc) / T(8);
    T c2 = g0 - mixT<T>(a, b, alpha);
    const T c2max = std::max(std::max(c2tl, c2tr), std::max(c2bl, c2br));
    const T c2min = std::min(std::min(c2tl, c2tr), std::min(c2bl, c2br));
    c2 = clampT<T>(c2, c2min, c2max);
    if (red) {
        out[0] = c1; out[1] = g0; out[2] = c2;
    } else {
        out[0] = c2; out[1] = g0; out[2] = c1;
    }
}

// interpolateRedBlueAtGreenPixel, demosaic.metal:422-499 (one G site).
template <class T>
inline void rb_at_g(const Plane4<T>& rgb, const Plane2<T>& grad, std::array<float, 2> rv, std::array<float, 2> bv, int x,
                    int y, T out[3]) {
    auto P = [&](int i, int j, int c) { return rgb.at(x + i, y + j, c); };
    const T g0 = P(0, 0, 1);
    const T lr = P(-1, 0, 0), lg = P(-1, 0, 1), lb = P(-1, 0, 2);
    const T rr = P(1, 0, 0), rg = P(1, 0, 1), rb = P(1, 0, 2);
    const T ur = P(0, -1, 0), ug = P(0, -1, 1), ub = P(0, -1, 2);
    const T dr = P(0, 1, 0), dg = P(0, 1, 1), db = P(0, 1, 2);
    const T red_ave = (lr + rr + ur + dr) / T(4);
    const T blue_ave = (lb + rb + ub + db) / T(4);
    const T gr_l = lg - lr, gr_r = rg - rr, gr_u = ug - ur, gr_d = dg - dr;
    const T gb_l = lg - lb, gb_r = rg - rb, gb_u = ug - ub, gb_d = dg - db;
    const T gr_l3 = P(-3, 0, 1) - P(-3, 0, 0), gr_r3 = P(3, 0, 1) - P(3, 0, 0);
    const T gr_u3 = P(0, -3, 1) - P(0, -3, 0), gr_d3 = P(0, 3, 1) - P(0, 3, 0);
    const T gb_l3 = P(-3, 0, 1) - P(-3, 0, 2), gb_r3 = P(3, 0, 1) - P(3, 0, 2);
    const T gb_u3 = P(0, -3, 1) - P(0, -3, 2), gb_d3 = P(0, 3, 1) - P(0, 3, 2);
    const T gx = std::abs(grad.at(x, y, 0)), gy = std::abs(grad.at(x, y, 1));
    const T dir = T(2) * std::atan2(gy, gx) / pi_v<T>();
    const T glen = std::sqrt(gx * gx + gy * gy);
    const T rsd = std::sqrt(T(rv[0]) + T(rv[1]) * red_ave);
    const T bsd = std::sqrt(T(bv[0]) + T(bv[1]) * blue_ave);
    const T ralpha = mixT<T>(T(0.5), dir, smoothstepT<T>(rsd, T(4) * rsd, glen));
    const T balpha = mixT<T>(T(0.5), dir, smoothstepT<T>(bsd, T(4) * bsd, glen));
    const T hl = T(1) - smoothstepT<T>(T(0.25), T(1), std::max(g0, std::max(std::max(rg, lg), std::max(dg, ug))));
    const T red = g0 - mixT<T>((gr_u + gr_d) / T(2) - hl * ((gr_d3 - gr_u) - (gr_d - gr_u3)) / T(8),
                               (gr_l + gr_r) / T(2) - hl * ((gr_r3 - gr_l) - (gr_r - gr_l3)) / T(8), ralpha);
    const T blue = g0 - mixT<T>((gb_u + gb_d) / T(2) - hl * ((gb_d3 - gb_u) - (gb_d - gb_u3)) / T(8),
                                (gb_l + gb_r) / T(2) - hl * ((gb_r3 - gb_l) - (gb_r - gb_l3)) / T(8), balpha);
    out[0] = clampT<T>(red, std::min(std::min(lr, rr), std::min(ur, dr)), std::max(std::max(lr, rr), std::max(ur, dr)));
    out[1] = g0;
    out[2] = clampT<T>(blue, std::min(std::min(lb, rb), std::min(ub, db)), std::max(std::max(lb, rb), std::max(ub, db)));
}

// demosaicImageKernel, demosaic_kernels.hpp:124-181: interpolateGreen ->
// interpolateRedBlue -> interpolateRedBlueAtGreen.
template <class T>
Plane4<T> demosaic(const Plane<T>& raw, const Plane2<T>& grad, int pattern,
                   const std::array<std::array<float, 2>, 3>& rawVar) {
    const Plane<T> green = interpolate_green(raw, grad, pattern, rawVar[1]);
    const int w = raw.w, h = raw.h;
    Plane4<T> tmp(w, h);  // interpolateRedBlue output, demosaic.metal:393-415
    const int (*off)[2] = kBayerOffsets[pattern];
    parallel_rows(h / 2, [&](int qy) {
        for (int qx = 0; qx < w / 2; qx++) {
            const int x0 = 2 * qx, y0 = 2 * qy;
            T o[3];
            rb_at_rb(raw, green, grad, rawVar[0], rawVar[2], true, x0 + off[0][0], y0 + off[0][1], o);
            T* p = tmp.px(x0 + off[0][0], y0 + off[0][1]);
            p[0] = o[0]; p[1] = o[1]; p[2] = o[2]; p[3] = 0;
            rb_at_rb(raw, green, grad, rawVar[0], rawVar[2], false, x0 + off[2][0], y0 + off[2][1], o);
            p = tmp.px(x0 + off[2][0], y0 + off[2][1]);
            p[0] = o[0]; p[1] = o[1]; p[2] = o[2]; p[3] = 0;
            for (int c : {1, 3}) {
                p = tmp.px(x0 + off[c][0], y0 + off[c][1]);
                p[0] = 0; p[1] = green.at(x0 + off[c][0], y0 + off[c][1]); p[2] = 0; p[3] = 0;
            }
        }
    });
    Plane4<T> out(w, h);  // interpolateRedBlueAtGreen, demosaic.metal:501-521
    parallel_rows(h / 2, [&](int qy) {
        for (int qx = 0; qx < w / 2; qx++) {
            const int x0 = 2 * qx, y0 = 2 * qy;
            for (int c : {1, 3}) {
                T o[3];
                const int x = x0 + off[c][0], y = y0 + off[c][1];
                rb_at_g(tmp, grad, rawVar[0], rawVar[2], x, y, o);
                T* p = out.px(x, y);
                p[0] = o[0]; p[1] = o[1]; p[2] = o[2]; p[3] = 0;
            }
            for (int c : {0, 2}) {
                const int x = x0 + off[c][0], y = y0 + off[c][1];
                std::memcpy(out.px(x, y), tmp.px(x, y), sizeof(T) * 4);
            }
        }
    });
    return out;
}

// blendHighlightsImage, demosaic.metal:536-564.
template <class T>
void blend_highlights(Plane4<T>& img, T clip) {
    static const T s3 = T(1.7320508f);
    const T tr[3][3] = {{1, 1, 1}, {s3, -s3, 0}, {-1, -1, 2}};
    const T itr[3][3] = {{1, s3 / T(2), T(-0.5)}, {1, -s3 / T(2), T(-0.5)}, {1, 0, 1}};
    parallel_rows(img.h, [&](int y) {
        for (int x = 0; x < img.w; x++) {
            T* p = img.px(x, y);
            if (!(p[0] > clip || p[1] > clip || p[2] > clip)) continue;
            T cam[2][3] = {{p[0], p[1], p[2]}, {std::min(p[0], clip), std::min(p[1], clip), std::min(p[2], clip)}};
            T lab[2][3], sum[2];
            for (int i = 0; i < 2; i++) {
                for (int r = 0; r < 3; r++) lab[i][r] = tr[r][0] * cam[i][0] + tr[r][1] * cam[i][1] + tr[r][2] * cam[i][2];
                sum[i] = lab[i][1] * lab[i][1] + lab[i][2] * lab[i][2];
            }
            const T chr = sum[0] > 0 ? std::sqrt(sum[1] / sum[0]) : T(1);
            lab[0][1] *= chr;
            lab[0][2] *= chr;
            for (int r = 0; r < 3; r++) p[r] = (itr[r][0] * lab[0][0] + itr[r][1] * lab[0][1] + itr[r][2] * lab[0][2]) / T(3);
        }
    });
}

// transformImage, demosaic.metal:649-662 (w channel written as 0).
template <class T>
void transform(Plane4<T>& img, const Mat3& m) {
    parallel_rows(img.h, [&](int y) {
        for (int x = 0; x < img.w; x++) {
            T* p = img.px(x, y);
            T v[3] = {p[0], p[1], p[2]};
            for (int r = 0; r < 3; r++) p[r] = T(m.m[r][0]) * v[0] + T(m.m[r][1]) * v[1] + T(m.m[r][2]) * v[2];
            p[3] = 0;
        }
    });
}

// despeckleLumaMedianChromaImage, demosaic.metal:1161-1283: luma clamped to
// the 2nd extrema of its 3x3 neighbourhood (noise gated), chroma 3x3 median.
template <class T>
Plane4<T> despeckle_luma_median_chroma(const Plane4<T>& in, const float var_a[3], const float var_b[3]) {
    Plane4<T> out(in.w, in.h);
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++) {
            T lum[9], cb[9], cr[9];
            int k = 0;
            for (int j = -1; j <= 1; j++)
                for (int i = -1; i <= 1; i++, k++) {
                    lum[k] = in.at(x + i, y + j, 0);
                    cb[k] = in.at(x + i, y + j, 1);
                    cr[k] = in.at(x + i, y + j, 2);
                }
            const T sample = lum[4];
            // top-2 / bottom-2 with the kernel's initial values (0 and +inf)
            T fmax = 0, smax = 0, fmin = INFINITY, smin = INFINITY;
            for (int i = 0; i < 9; i++) {
                const T v = lum[i];
                smax = (v <= fmax && v > smax) ? v : smax;
                smax = v > fmax ? fmax : smax;
                fmax = v > fmax ? v : fmax;
                smin = (v >= fmin && v < smin) ? v : smin;
                smin = v < fmin ? fmin : smin;
                fmin = v < fmin ? v : fmin;
            }
            std::nth_element(cb, cb + 4, cb + 9);
            std::nth_element(cr, cr + 4, cr + 9);
            const T sigma = std::sqrt(T(var_a[0]) + T(var_b[0]) * sample);
            const T minv = mixT<T>(smin, fmin, smoothstepT<T>(sigma, T(4) * sigma, smin - fmin));
            const T maxv = mixT<T>(smax, fmax, smoothstepT<T>(sigma, T(4) * sigma, fmax - smax));
            T* o = out.px(x, y);
            o[0] = clampT<T>(sample, minv, maxv);
            o[1] = cb[4];
            o[2] = cr[4];
            o[3] = 0;
        }
    });
    return out;
}

// ---- high-noise raw branch (raw_converter.cpp:195-202) ----

// bayerToRawRGBA, demosaic.metal:961-978: quad -> (R, G, B, G2).
template <class T>
Plane4<T> bayer_to_rgba(const Plane<T>& raw, int pattern) {
    Plane4<T> out(raw.w / 2, raw.h / 2);
    const int (*off)[2] = kBayerOffsets[pattern];
    parallel_rows(out.h, [&](int y) {
        for (int x = 0; x < out.w; x++)
            for (int c = 0; c < 4; c++) out.px(x, y)[c] = raw.at(2 * x + off[c][0], 2 * y + off[c][1]);
    });
    return out;
}

// rawRGBAToBayer, demosaic.metal:980-997.
template <class T>
void rgba_to_bayer(const Plane4<T>& rgba, int pattern, Plane<T>& raw) {
    const int (*off)[2] = kBayerOffsets[pattern];
    parallel_rows(rgba.h, [&](int y) {
        for (int x = 0; x < rgba.w; x++)
            for (int c = 0; c < 4; c++) raw.px(2 * x + off[c][0], 2 * y + off[c][1])[0] = rgba.px(x, y)[c];
    });
}

// despeckleRawRGBAImage + despeckle_3x3x4, demosaic.metal:1025-1092.
template <class T>
Plane4<T> despeckle_raw_rgba(const Plane4<T>& in, const Plane2<T>& grad, const float var[4]) {
    Plane4<T> out(in.w, in.h);
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++) {
            const T g0 = grad.at(2 * x, 2 * y, 0), g1 = grad.at(2 * x, 2 * y, 1);
            const T gradient = std::sqrt(g0 * g0 + g1 * g1);
            for (int c = 0; c < 4; c++) {
                T fmax = 0, smax = 0, fmin = T(65504), smin = T(65504);
                for (int i = -1; i <= 1; i++)
                    for (int j = -1; j <= 1; j++) {
                        const T v = in.at(x + i, y + j, c);
                        smax = v >= fmax ? fmax : std::max(v, smax);
                        fmax = std::max(v, fmax);
                        smin = v <= fmin ? fmin : std::min(v, smin);
                        fmin = std::min(v, fmin);
                    }
                const T s = in.at(x, y, c);
                const T sigma = std::sqrt(T(var[c]) * s);
                const T tex = T(1) - T(0.5) * smoothstepT<T>(T(1), T(2), gradient / sigma);
                const T minv = mixT<T>(fmin, smin, tex * (T(1) - smoothstepT<T>(T(2) * sigma, T(8) * sigma, smin - fmin)));
                const T maxv = mixT<T>(fmax, smax, tex * (T(1) - smoothstepT<T>(sigma, T(4) * sigma, fmax - smax)));
                out.px(x, y)[c] = clampT<T>(s, minv, maxv);
            }
        }
    });
    return out;
}

// crossDenoiseRawRGBAImage, demosaic.metal:999-1023: 5x5 bilateral on quads.
template <class T>
Plane4<T> cross_denoise_raw_rgba(const Plane4<T>& in, const float var[4], float strength) {
    Plane4<T> out(in.w, in.h);
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++) {
            const T* p = in.px(x, y);
            T inv[4];
            for (int c = 0; c < 4; c++) inv[c] = T(1) / (T(strength) * std::sqrt(T(var[c]) * (p[c] + T(0.0001))));
            T sum[4] = {0, 0, 0, 0}, sw = 0;
            for (int j = -2; j <= 2; j++)
                for (int i = -2; i <= 2; i++) {
                    T s[4], d2 = 0;
                    for (int c = 0; c < 4; c++) {
                        s[c] = in.at(x + i, y + j, c);
                        const T d = (p[c] - s[c]) * inv[c];
                        d2 += d * d;
                    }
                    const T w = std::exp(T(-2) * d2);
                    for (int c = 0; c < 4; c++) sum[c] += w * s[c];
                    sw += w;
                }
            for (int c = 0; c < 4; c++) out.px(x, y)[c] = sum[c] / sw;
        }
    });
    return out;
}

// ---- pyramid (pyramid_processor.cpp:96-172) ----

// downsampleImageXYZ / XY, demosaic.metal:886-920: mean of four bilinear
// samples at output texel centre +- half an output texel.
template <class T, int C>
Img<T, C> downsample(const Img<T, C>& in, int ow, int oh, int nch) {
    Img<T, C> out(ow, oh);
    const T rx = T(in.w) / T(ow), ry = T(in.h) / T(oh);
    parallel_rows(oh, [&](int y) {
        for (int x = 0; x < ow; x++) {
            const T u0 = T(x) * rx - T(0.5), u1 = (T(x) + T(1)) * rx - T(0.5);
            const T v0 = T(y) * ry - T(0.5), v1 = (T(y) + T(1)) * ry - T(0.5);
            for (int c = 0; c < nch; c++) {
                T s = in.bilin(u0, v0, c) + in.bilin(u1, v0, c) + in.bilin(u0, v1, c) + in.bilin(u1, v1, c);
                out.px(x, y)[c] = T(0.25) * s;
            }
        }
    });
    return out;
}

// subtractNoiseImage, demosaic.metal:922-959 (reconstruct step).
template <class T>
Plane4<T> subtract_noise(const Plane4<T>& in, const Plane4<T>& coarse, const Plane4<T>& coarse_den,
                         const Plane2<T>& grad, float luma_weight, float sharpening, float nlf_a, float nlf_b) {
    Plane4<T> out(in.w, in.h);
    const T rx = T(coarse.w) / T(in.w), ry = T(coarse.h) / T(in.h);
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++) {
            const T u = (T(x) + T(0.5)) * rx - T(0.5), v = (T(y) + T(0.5)) * ry - T(0.5);
            const T* ip = in.px(x, y);
            T p1[3], pd[3], dn[3];
            for (int c = 0; c < 3; c++) {
                p1[c] = coarse.bilin(u, v, c);
                pd[c] = coarse_den.bilin(u, v, c);
                dn[c] = ip[c] - (c == 0 ? T(luma_weight) : T(1)) * (p1[c] - pd[c]);
            }
            T alpha = T(sharpening);
            if (sharpening > 1.0f) {
                const T g0 = grad.at(x, y, 0), g1 = grad.at(x, y, 1);
                const T gm = std::sqrt(g0 * g0 + g1 * g1);
                const T sigma = std::sqrt(T(nlf_a) + T(nlf_b) * pd[0]);
                const T detail = smoothstepT<T>(sigma, T(4) * sigma, gm) * (T(1) - smoothstepT<T>(T(0.75), T(0.95), pd[0])) *
                                 smoothstepT<T>(T(0.05), T(0.1), pd[0]);
                alpha = T(1) + (alpha - T(1)) * detail;
            }
            T* o = out.px(x, y);
            for (int c = 0; c < 3; c++) o[c] = mixT<T>(pd[c], dn[c], alpha);
            o[0] = std::max(o[0], T(0));
            o[3] = ip[3];
        }
    });
    return out;
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (double).
// Replaces Eigen::SelfAdjointEigenSolver (PCA.cpp:36). On return a's
// diagonal holds the eigenvalues and v's columns the eigenvectors.
inline void jacobi_eigen(int n, std::vector<double>& a, std::vector<double>& v) {
    v.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; i++) v[i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += a[i * n + j] * a[i * n + j];
                if (i != j) off += a[i * n + j] * a[i * n + j];
            }
        if (off <= 1e-26 * tot || off == 0) break;  // off-diagonal norm <= 1e-13 x total
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = a[p * n + q];
                if (std::abs(apq) < 1e-300) continue;
                const double app = a[p * n + p], aqq = a[q * n + q];
                const double theta = (aqq - app) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; k++) {  // rotate columns p, q
                    const double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = c * akp - s * akq;
                    a[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {  // rotate rows p, q
                    const double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = c * apk - s * aqk;
                    a[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    const double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = c * vkp - s * vkq;
                    v[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
}

// Top-8 basis from eigenpairs sorted by decreasing eigenvalue (ev[c], column
// c of evec). Eigenvectors whose eigenvalue is not above 1e-9 x the largest
// (a rank-deficient sample: fewer than 26 patches, or a flat image) span a
// null space whose basis any solver picks arbitrarily; those columns are
// instead completed deterministically by Gram-Schmidt of the unit vectors
// e0, e1, ... against the columns before them. Every column's sign is fixed
// so that its largest-magnitude entry (first on ties) is positive.
inline void select_basis(const double ev[25], const double evec[25][25], std::array<std::array<double, 8>, 25>& basis) {
    const double lam0 = std::max(ev[0], double(0));
    const double tol = 1e-9 * lam0;
    int cand = 0;
    bool kept = true;
    for (int c = 0; c < 8; c++) {
        double v[25];
        kept = kept && lam0 > 0 && ev[c] > tol;
        if (kept) {
            for (int r = 0; r < 25; r++) v[r] = evec[r][c];
        } else {
            for (;;) {
                for (int r = 0; r < 25; r++) v[r] = (r == cand) ? 1.0 : 0.0;
                cand++;
                for (int pass = 0; pass < 2; pass++)
                    for (int k = 0; k < c; k++) {
                        double d = 0;
                        for (int r = 0; r < 25; r++) d += basis[r][k] * v[r];
                        for (int r = 0; r < 25; r++) v[r] -= d * basis[r][k];
                    }
                double nn = 0;
                for (int r = 0; r < 25; r++) nn += v[r] * v[r];
                if (nn > 0.25) {
                    const double inv = 1.0 / std::sqrt(nn);
                    for (int r = 0; r < 25; r++) v[r] *= inv;
                    break;
                }
            }
        }
        int amax = 0;
        for (int r = 1; r < 25; r++)
            if (std::abs(v[r]) > std::abs(v[amax])) amax = r;
        const double sgn = v[amax] < 0 ? -1.0 : 1.0;
        for (int r = 0; r < 25; r++) basis[r][c] = sgn * v[r];
    }
}

// collectPatches + build_pca_space<25, 8>, demosaic.metal:755-772 and
// PCA.cpp:23-56: 5x5 luma patches on the 8-pixel grid, mean-centred
// covariance / (n - 1) (accumulated in double), top-8 eigenvectors in
// decreasing eigenvalue order (select_basis). Fewer than 2 patches: the
// first 8 unit vectors.
template <class T>
std::array<std::array<double, 8>, 25> pca_basis(const Plane4<T>& img) {
    const int gw = img.w / 8, gh = img.h / 8;
    const int n = gw * gh;
    std::array<std::array<double, 8>, 25> basis{};
    if (n < 2) {
        for (int r = 0; r < 25; r++)
            for (int c = 0; c < 8; c++) basis[r][c] = (r == c) ? 1.0 : 0.0;
        return basis;
    }
    std::vector<double> patches(size_t(n) * 25);
    for (int y = 0; y < gh; y++)
        for (int x = 0; x < gw; x++)
            for (int j = -2; j <= 2; j++)
                for (int i = -2; i <= 2; i++)
                    patches[size_t(y * gw + x) * 25 + (j + 2) * 5 + (i + 2)] = double(img.at(8 * x + i, 8 * y + j, 0));
    double mean[25] = {0};
    for (int k = 0; k < n; k++)
        for (int r = 0; r < 25; r++) mean[r] += patches[size_t(k) * 25 + r];
    for (int r = 0; r < 25; r++) mean[r] /= n;
    std::vector<double> cov(25 * 25, 0.0);
    for (int k = 0; k < n; k++) {
        double d[25];
        for (int r = 0; r < 25; r++) d[r] = patches[size_t(k) * 25 + r] - mean[r];
        for (int r = 0; r < 25; r++)
            for (int c = r; c < 25; c++) cov[r * 25 + c] += d[r] * d[c];
    }
    for (int r = 0; r < 25; r++)
        for (int c = r; c < 25; c++) {
            cov[r * 25 + c] /= (n - 1);
            cov[c * 25 + r] = cov[r * 25 + c];
        }
    std::vector<double> vec;
    jacobi_eigen(25, cov, vec);
    int idx[25];
    for (int i = 0; i < 25; i++) idx[i] = i;
    std::stable_sort(idx, idx + 25, [&](int a, int b) { return cov[a * 25 + a] > cov[b * 25 + b]; });
    double ev[25], evec[25][25];
    for (int c = 0; c < 25; c++) {
        ev[c] = cov[idx[c] * 25 + idx[c]];
        for (int r = 0; r < 25; r++) evec[r][c] = vec[r * 25 + idx[c]];
    }
    select_basis(ev, evec, basis);
    return basis;
}

// pcaProjection, demosaic.metal:774-796: 5x5 luma patch x basis -> 8 coefs.
template <class T>
Img<T, 8> pca_project(const Plane4<T>& img, const std::array<std::array<double, 8>, 25>& basis) {
    Img<T, 8> out(img.w, img.h);
    T b[25][8];
    for (int r = 0; r < 25; r++)
        for (int c = 0; c < 8; c++) b[r][c] = T(basis[r][c]);
    parallel_rows(img.h, [&](int y) {
        for (int x = 0; x < img.w; x++) {
            T acc[8] = {0};
            int row = 0;
            for (int j = -2; j <= 2; j++)
                for (int i = -2; i <= 2; i++, row++) {
                    const T v = img.at(x + i, y + j, 0);
                    for (int c = 0; c < 8; c++) acc[c] += b[row][c] * v;
                }
            for (int c = 0; c < 8; c++) out.px(x, y)[c] = acc[c];
        }
    });
    return out;
}

// blockMatchingDenoiseImage, demosaic.metal:806-884: 21x21 non-local means
// with PCA-space patch distance for luma, chroma distance for chroma and a
// fixed spatial Gaussian. Output (Y, Cb, Cr, luma kernel norm).
template <class T>
Plane4<T> block_match(const Plane4<T>& img, const Plane2<T>& grad, const Img<T, 8>& pca, const YCbCrNLF& nlf,
                      const DenoiseParams& dp, float lsc) {
    Plane4<T> out(img.w, img.h);
    const T cx = T(img.w / 2), cy = T(img.h / 2);
    const T clen = std::sqrt(cx * cx + cy * cy);
    T spatial[21][21];
    for (int y = -10; y <= 10; y++)
        for (int x = -10; x <= 10; x++) spatial[y + 10][x + 10] = gaussianT<T>(T(0.1) * std::sqrt(T(x * x + y * y)));
    const T tm[3] = {T(dp.luma), T(dp.chroma), T(dp.chroma)};
    parallel_rows(img.h, [&](int y) {
        for (int x = 0; x < img.w; x++) {
            const T* in = img.px(x, y);
            const T* ip = pca.px(x, y);
            T ls = 1;
            if (lsc > 0) {
                const T dx = T(x) - cx, dy = T(y) - cy;
                const T r = std::sqrt(dx * dx + dy * dy) / clen;
                ls = T(1) + T(lsc) * r * r;
            }
            T dm[3];
            for (int c = 0; c < 3; c++) dm[c] = T(1) / (tm[c] * std::sqrt(T(nlf.a[c]) + T(nlf.b[c]) * ls * in[0]));
            const T g0 = grad.at(x, y, 0), g1 = grad.at(x, y, 1);
            const T mag = std::sqrt(g0 * g0 + g1 * g1);
            const T sigma0 = std::sqrt(T(nlf.a[0]) + T(nlf.b[0]) * ls * in[0]);
            const T edge = smoothstepT<T>(T(2), T(16), T(dp.gradientThreshold) * mag / sigma0);
            const T lscale = dm[0] / (T(1) + T(dp.gradientBoost) * edge);
            const T cscale1 = dm[1] / T(dp.chromaBoost), cscale2 = dm[2] / T(dp.chromaBoost);
            T fy = 0, fcb = 0, fcr = 0, ny = 0, nc = 0;
            for (int j = -10; j <= 10; j++)
                for (int i = -10; i <= 10; i++) {
                    const int sx = std::clamp(x + i, 0, img.w - 1), sy = std::clamp(y + j, 0, img.h - 1);
                    const T* s = img.px(sx, sy);
                    const T* sp = pca.px(sx, sy);
                    T d2 = 0;
                    for (int c = 0; c < 8; c++) {
                        const T d = sp[c] - ip[c];
                        d2 += d * d;
                    }
                    const T ld = std::sqrt(d2) * lscale;
                    const T lw = std::exp(T(-2) * ld * ld);
                    const T c1 = (s[1] - in[1]) * cscale1, c2 = (s[2] - in[2]) * cscale2;
                    const T cw = std::exp(T(-2) * (lw * lw + c1 * c1 + c2 * c2));
                    const T sw = spatial[j + 10][i + 10];
                    const T wy = sw * lw, wc = sw * cw;
                    fy += wy * s[0];
                    fcb += wc * s[1];
                    fcr += wc * s[2];
                    ny += wy;
                    nc += wc;
                }
            T* o = out.px(x, y);
            o[0] = fy / ny;
            o[1] = fcb / nc;
            o[2] = fcr / nc;
            o[3] = ny;
        }
    });
    return out;
}

struct PyramidOut {
    std::vector<std::array<std::array<double, 8>, 25>> bases;
};

// PyramidProcessor<levels>::denoise, pyramid_processor.cpp:96-172.
// frozen (optional): per-level PCA bases to use instead of computing them
// (the adjoint's gradient checks hold the bases fixed).
template <class T>
Plane4<T> pyramid_denoise(const Plane4<T>& image, const Plane2<T>& gradient, const Params& p,
                          std::vector<Plane4<T>>* denoised_levels = nullptr, PyramidOut* info = nullptr,
                          const std::vector<std::array<std::array<double, 8>, 25>>* frozen = nullptr) {
    const int L = p.levels;
    std::vector<Plane4<T>> img(L);     // img[i] = level i input (img[0] = image)
    std::vector<Plane2<T>> grad(L);
    img[0] = image;
    grad[0] = gradient;
    for (int i = 1; i < L; i++) {
        const int w = image.w >> i, h = image.h >> i;  // width / 2^i (floor), :38-41
        img[i] = downsample<T, 4>(img[i - 1], w, h, 3);
        grad[i] = downsample<T, 2>(grad[i - 1], w, h, 2);
    }
    static const float lumaDenoiseWeight[4] = {1, 1, 1, 1};  // :93
    std::vector<Plane4<T>> den(L);
    if (info) info->bases.assign(L, {});
    for (int i = L - 1; i >= 0; i--) {
        const DenoiseParams& dp = p.dn[i];
        Plane4<T> layer;
        if (i < L - 1) {
            const float na = p.pyr_nlf[i].a[0] * dp.luma, nb = p.pyr_nlf[i].b[0] * dp.luma;
            layer = subtract_noise(img[i], img[i + 1], den[i + 1], grad[i], lumaDenoiseWeight[i], dp.sharpening, na, nb);
        } else {
            layer = img[i];
        }
        const auto basis = frozen ? (*frozen)[i] : pca_basis(layer);
        if (info) info->bases[i] = basis;
        const auto pca = pca_project(layer, basis);
        den[i] = block_match(layer, grad[i], pca, p.pyr_nlf[i], dp, p.lsc);
    }
    if (denoised_levels) *denoised_levels = den;
    return den[0];
}

struct Stages {
    bool keep = false;
    Plane<float> scaled;     // filled when keep (converted to float)
    Plane2<float> gradient;
    Plane4<float> demosaiced;
    Plane4<float> despeckled;
};

template <class T, int C>
Img<float, C> to_float(const Img<T, C>& a) {
    Img<float, C> r(a.w, a.h);
    for (size_t i = 0; i < a.d.size(); i++) r.d[i] = float(a.d[i]);
    return r;
}

// RawConverter::demosaic, raw_converter.cpp:148-248, without
// post-processing (linear camera RGB out, RGBA with w = 0).
template <class T>
Plane4<T> raw_pipeline(const uint16_t* raw, size_t stride_elems, int w, int h, const Params& p, bool denoise,
                       Stages* st = nullptr, PyramidOut* info = nullptr) {
    static const Taps t1 = gaussian_bilinear_taps(1.5f), t2 = gaussian_bilinear_taps(4.5f);
    Plane<T> scaled = scale_raw<T>(raw, stride_elems, w, h, p);
    const Plane4<T> sob = sobel(scaled);
    const auto rv = raw_variance(p.raw_nlf);
    const Plane2<T> grad = gradient_blur(scaled, sob, t1, t2, rv[1]);
    if (denoise && p.high_noise) {
        Plane4<T> rgba = bayer_to_rgba(scaled, p.bayer);
        Plane4<T> ds = despeckle_raw_rgba(rgba, grad, p.raw_nlf.b);
        Plane4<T> cd = cross_denoise_raw_rgba(ds, p.raw_nlf.b, p.raw_strength);
        rgba_to_bayer(cd, p.bayer, scaled);
    }
    Plane4<T> rgb = demosaic(scaled, grad, p.bayer, rv);
    blend_highlights(rgb, T(1));
    if (st && st->keep) {
        st->scaled = to_float(scaled);
        st->gradient = to_float(grad);
        st->demosaiced = to_float(rgb);
    }
    if (!denoise) return rgb;
    const Mat3 c2y = cam_ycbcr(p.rgb_cam, p.xyz_rgb);
    const Mat3 y2c = inverse3(c2y);
    transform(rgb, c2y);
    Plane4<T> ds = despeckle_luma_median_chroma(rgb, p.pyr_nlf[0].a, p.pyr_nlf[0].b);
    if (st && st->keep) st->despeckled = to_float(ds);
    Plane4<T> den = pyramid_denoise<T>(ds, grad, p, nullptr, info);
    transform(den, y2c);
    return den;
}

}  // namespace orc
