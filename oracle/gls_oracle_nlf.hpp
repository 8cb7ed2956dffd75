// gls_oracle_nlf.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the
// reference's noise-model measurement (RawConverter with calibrateFromImage),
// the checker for the CUDA kernels in gls_nlf.cu:
//   * raw_stats   basicRawNoiseStatistics, demosaic.metal:1110-1136
//   * ycc_stats   basicNoiseStatistics, demosaic.metal:1138-1159
//   * measure_raw RawConverter::MeasureRawNLF, raw_converter.cpp:339-490
//   * measure_ycc PyramidProcessor::MeasureYCbCrNLF, pyramid_processor.cpp:173-324
// Statistics in T (float reproduces the reference's texture2d<float>
// kernels operation for operation); the regressions in double, summed over
// the statistics images row by row as the reference's image apply() does.
// Pinned against the reference's own kernels and regressions compiled for
// the CPU (oracle/ref_harness.cpp, oracle/ref_nlf.cpp).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>

#include "gls_oracle.hpp"

namespace orc {
namespace nlf {

// 9x9 window statistics of the four raw channels at every half-resolution
// position. The window steps one full-resolution pixel at a time from
// 2 * (x, y), and at each step reads the quad at that position plus each
// channel's Bayer offset (readRAWQuad, demosaic.metal:1094-1107), so a step
// with an odd offset reads its neighbours' channels, as the reference does.
// Reads clamp to the frame.
template <class T>
inline void raw_stats(const Plane<T>& scaled, int bayer, Plane4<T>& mean, Plane4<T>& var) {
    const int W2 = scaled.w / 2, H2 = scaled.h / 2;
    mean = Plane4<T>(W2, H2);
    var = Plane4<T>(W2, H2);
    const auto& off = kBayerOffsets[bayer];
    parallel_rows(H2, [&](int y) {
        for (int x = 0; x < W2; x++) {
            const T count = T(81);
            T sum[4] = {0, 0, 0, 0}, sumSq[4] = {0, 0, 0, 0};
            for (int dy = -4; dy <= 4; dy++)
                for (int dx = -4; dx <= 4; dx++) {
                    const int bx = 2 * x + dx, by = 2 * y + dy;
                    for (int c = 0; c < 4; c++) {
                        const T s = scaled.at(bx + off[c][0], by + off[c][1]);
                        sum[c] = sum[c] + s;
                        sumSq[c] = sumSq[c] + s * s;
                    }
                }
            for (int c = 0; c < 4; c++) {
                mean.px(x, y)[c] = sum[c] / count;
                var.px(x, y)[c] = (sumSq[c] - (sum[c] * sum[c]) / count) / count;
            }
        }
    });
}

// 5x5 window statistics of a YCbCr level: (mean Y, var Y, var Cb, var Cr)
template <class T>
inline Plane4<T> ycc_stats(const Plane4<T>& img) {
    Plane4<T> st(img.w, img.h);
    parallel_rows(img.h, [&](int y) {
        for (int x = 0; x < img.w; x++) {
            const T count = T(25);
            T sum[3] = {0, 0, 0}, sumSq[3] = {0, 0, 0};
            for (int dy = -2; dy <= 2; dy++)
                for (int dx = -2; dx <= 2; dx++)
                    for (int c = 0; c < 3; c++) {
                        const T s = img.at(x + dx, y + dy, c);
                        sum[c] = sum[c] + s;
                        sumSq[c] = sumSq[c] + s * s;
                    }
            T* o = st.px(x, y);
            o[0] = sum[0] / count;
            for (int c = 0; c < 3; c++) o[1 + c] = (sumSq[c] - (sum[c] * sum[c]) / count) / count;
        }
    });
    return st;
}

// the variance class of the largest component: 6 + trunc(clamp(log10, -6,
// -1)), the largest taken from the first component on (a NaN in a later
// component never wins). A NaN largest value (a negative variance in the
// first channel, from rounding in a flat region) has no class: the
// reference converts it to an int, which indexes outside its six-entry
// histogram (undefined), so here it is not counted (-1).
template <int N>
inline int variance_class(const double (&v)[N]) {
    double m = std::log10(v[0]);
    for (int i = 1; i < N; i++) {
        const double l = std::log10(v[i]);
        if (l > m) m = l;
    }
    if (std::isnan(m)) return -1;
    return 6 + int(std::clamp(m, -6.0, -1.0));
}

// max(v, s) of the reference's vector type: v where v > s, else s (so a NaN
// fit falls back to s)
inline double max_s(double v, double s) { return v > s ? v : s; }

// the variance bound from the class histogram (raw_converter.cpp:364-369)
inline double variance_bound(const double hist[6]) {
    return hist[0] > 1e3 ? 1.0e-5 : hist[1] > 1e3 ? 1.0e-4 : hist[2] > 1e3 ? 1.0e-3
         : hist[3] > 1e3 ? 1.0e-2 : hist[4] > 1e3 ? 1.0e-1 : 1;
}

// MeasureRawNLF over the statistics images: the variance bound from the
// histogram of variance classes; a least-squares line var = A + B mean per
// channel over positions with every channel's mean in [0.001, 0.9] and
// variance under the bound; then a second fit over positions within the
// bound B whose squared residuals are all <= half the first fit's mean
// squared residual, kept if it covers more than 0.1% of the raw pixels and
// its mean squared residual is below the first's in every channel. A and B
// are floored at 1e-8 and scaled by exposure_multiplier^2.
template <class T>
inline RawNLF measure_raw(const Plane4<T>& mean, const Plane4<T>& var, int raw_w, int raw_h,
                          float exposure_multiplier) {
    using D4 = std::array<double, 4>;
    auto isnan4 = [](const double* v) { return std::isnan(v[0]) || std::isnan(v[1]) || std::isnan(v[2]) || std::isnan(v[3]); };
    auto load = [](const T* p, double* v) {
        for (int c = 0; c < 4; c++) v[c] = double(float(p[c]));
    };
    double hist[6] = {0, 0, 0, 0, 0, 0};
    for (int y = 0; y < var.h; y++)
        for (int x = 0; x < var.w; x++) {
            double v[4];
            load(var.px(x, y), v);
            if (!isnan4(v)) {
                const int k = variance_class<4>(v);
                if (k >= 0) hist[k]++;
            }
        }
    D4 vmax;
    vmax.fill(variance_bound(hist));
    const double maxValue = 0.9, minValue = 0.001;
    auto in_range = [&](const double* m, const double* v, const D4& bound) {
        if (isnan4(m) || isnan4(v)) return false;
        for (int c = 0; c < 4; c++)
            if (!(m[c] >= minValue) || !(m[c] <= maxValue) || !(v[c] <= bound[c])) return false;
        return true;
    };
    D4 sx{}, sy{}, sxx{}, sxy{};
    double N1 = 0;
    for (int y = 0; y < mean.h; y++)
        for (int x = 0; x < mean.w; x++) {
            double m[4], v[4];
            load(mean.px(x, y), m);
            load(var.px(x, y), v);
            if (in_range(m, v, vmax)) {
                for (int c = 0; c < 4; c++) {
                    sx[c] += m[c];
                    sy[c] += v[c];
                    sxx[c] += m[c] * m[c];
                    sxy[c] += m[c] * v[c];
                }
                N1++;
            }
        }
    D4 A, B;
    for (int c = 0; c < 4; c++) {
        B[c] = max_s((N1 * sxy[c] - sx[c] * sy[c]) / (N1 * sxx[c] - sx[c] * sx[c]), 1e-8);
        A[c] = max_s((sy[c] - B[c] * sx[c]) / N1, 1e-8);
    }
    D4 err2{};
    for (int y = 0; y < mean.h; y++)
        for (int x = 0; x < mean.w; x++) {
            double m[4], v[4];
            load(mean.px(x, y), m);
            load(var.px(x, y), v);
            if (in_range(m, v, vmax))
                for (int c = 0; c < 4; c++) {
                    const double d = (A[c] + B[c] * m[c]) - v[c];
                    err2[c] += d * d;
                }
        }
    for (int c = 0; c < 4; c++) err2[c] /= N1;
    vmax = B;
    D4 newErr2{};
    sx = sy = sxx = sxy = D4{};
    double N2 = 0;
    for (int y = 0; y < mean.h; y++)
        for (int x = 0; x < mean.w; x++) {
            double m[4], v[4];
            load(mean.px(x, y), m);
            load(var.px(x, y), v);
            if (!in_range(m, v, vmax)) continue;
            double d2[4];
            bool fits = true;
            for (int c = 0; c < 4; c++) {
                const double d = std::abs((A[c] + B[c] * m[c]) - v[c]);
                d2[c] = d * d;
                fits = fits && d2[c] <= 0.5 * err2[c];
            }
            if (fits) {
                for (int c = 0; c < 4; c++) {
                    sx[c] += m[c];
                    sy[c] += v[c];
                    sxx[c] += m[c] * m[c];
                    sxy[c] += m[c] * v[c];
                    newErr2[c] += d2[c];
                }
                N2++;
            }
        }
    for (int c = 0; c < 4; c++) newErr2[c] /= N2;
    bool better = !(std::isnan(newErr2[0]) || std::isnan(newErr2[1]) || std::isnan(newErr2[2]) || std::isnan(newErr2[3]));
    for (int c = 0; c < 4; c++) better = better && newErr2[c] < err2[c];
    if (N2 > 0.001 * (raw_w * raw_h) && better) {
        for (int c = 0; c < 4; c++) {
            B[c] = max_s((N2 * sxy[c] - sx[c] * sy[c]) / (N2 * sxx[c] - sx[c] * sx[c]), 1e-8);
            A[c] = max_s((sy[c] - B[c] * sx[c]) / N2, 1e-8);
        }
    }
    const double adj = exposure_multiplier * exposure_multiplier;  // a float product, as in the reference
    RawNLF r;
    for (int c = 0; c < 4; c++) {
        r.a[c] = float(A[c] * adj);
        r.b[c] = float(B[c] * adj);
    }
    return r;
}

// MeasureYCbCrNLF over one level's statistics: the same two-pass fit with
// the luma mean as the regressor of all three variances, positions with a
// positive variance in every channel for the class histogram, the second
// pass keeping squared residuals <= the first fit's mean squared residual,
// accepted if its mean squared residual is <= the first's in every channel
// and it covers more than 1% of the level.
template <class T>
inline YCbCrNLF measure_ycc(const Plane4<T>& st, float exposure_multiplier) {
    using D3 = std::array<double, 3>;
    auto isnan3 = [](const double* v) { return std::isnan(v[0]) || std::isnan(v[1]) || std::isnan(v[2]); };
    double hist[6] = {0, 0, 0, 0, 0, 0};
    for (int y = 0; y < st.h; y++)
        for (int x = 0; x < st.w; x++) {
            const T* p = st.px(x, y);
            const double v[3] = {double(float(p[1])), double(float(p[2])), double(float(p[3]))};
            if (!isnan3(v) && v[0] > 0.0 && v[1] > 0.0 && v[2] > 0.0) hist[variance_class<3>(v)]++;  // log10 finite
        }
    D3 vmax;
    vmax.fill(variance_bound(hist));
    const double maxValue = 0.9, minValue = 0.001;
    auto usable = [&](double m, const double* v, const D3& bound) {
        if (std::isnan(m) || isnan3(v)) return false;
        return m >= minValue && m <= maxValue && v[0] <= bound[0] && v[1] <= bound[1] && v[2] <= bound[2];
    };
    double sx = 0, sxx = 0, N = 0;
    D3 sy{}, sxy{};
    for (int y = 0; y < st.h; y++)
        for (int x = 0; x < st.w; x++) {
            const T* p = st.px(x, y);
            const double m = double(float(p[0]));
            const double v[3] = {double(float(p[1])), double(float(p[2])), double(float(p[3]))};
            if (usable(m, v, vmax)) {
                sx += m;
                for (int c = 0; c < 3; c++) sy[c] += v[c];
                sxx += m * m;
                for (int c = 0; c < 3; c++) sxy[c] += m * v[c];
                N++;
            }
        }
    D3 A, B;
    for (int c = 0; c < 3; c++) {
        B[c] = max_s((N * sxy[c] - sx * sy[c]) / (N * sxx - sx * sx), 1e-8);
        A[c] = max_s((sy[c] - B[c] * sx) / N, 1e-8);
    }
    D3 err2{};
    for (int y = 0; y < st.h; y++)
        for (int x = 0; x < st.w; x++) {
            const T* p = st.px(x, y);
            const double m = double(float(p[0]));
            const double v[3] = {double(float(p[1])), double(float(p[2])), double(float(p[3]))};
            if (usable(m, v, vmax))
                for (int c = 0; c < 3; c++) {
                    const double d = (A[c] + B[c] * m) - v[c];
                    err2[c] += d * d;
                }
        }
    for (int c = 0; c < 3; c++) err2[c] /= N;
    vmax = B;
    sx = sxx = N = 0;
    sy = sxy = D3{};
    D3 newErr2{};
    for (int y = 0; y < st.h; y++)
        for (int x = 0; x < st.w; x++) {
            const T* p = st.px(x, y);
            const double m = double(float(p[0]));
            const double v[3] = {double(float(p[1])), double(float(p[2])), double(float(p[3]))};
            if (!usable(m, v, vmax)) continue;
            double d2[3];
            bool fits = true;
            for (int c = 0; c < 3; c++) {
                const double d = std::abs((A[c] + B[c] * m) - v[c]);
                d2[c] = d * d;
                fits = fits && d2[c] <= err2[c];
            }
            if (fits) {
                sx += m;
                for (int c = 0; c < 3; c++) sy[c] += v[c];
                sxx += m * m;
                for (int c = 0; c < 3; c++) sxy[c] += m * v[c];
                N++;
                for (int c = 0; c < 3; c++) newErr2[c] += d2[c];
            }
        }
    for (int c = 0; c < 3; c++) newErr2[c] /= N;
    const bool better = newErr2[0] <= err2[0] && newErr2[1] <= err2[1] && newErr2[2] <= err2[2];
    if (better && N / (st.w * st.h) > 0.01) {
        for (int c = 0; c < 3; c++) {
            B[c] = max_s((N * sxy[c] - sx * sy[c]) / (N * sxx - sx * sx), 1e-8);
            A[c] = max_s((sy[c] - B[c] * sx) / N, 1e-8);
        }
    }
    const double adj = exposure_multiplier * exposure_multiplier;  // a float product, as in the reference
    YCbCrNLF r;
    for (int c = 0; c < 3; c++) {
        r.a[c] = float(A[c] * adj);
        r.b[c] = float(B[c] * adj);
    }
    return r;
}

}  // namespace nlf
}  // namespace orc

namespace orc {
namespace nlf {

// RawConverter::demosaic with calibrateFromImage (raw_converter.cpp:148-248,
// pyramid_processor.cpp:96-117): the raw noise model measured on the scaled
// frame replaces the given one before the gradient blur, the high-noise
// branch is off, despeckling uses the given level-0 pyramid model, and each
// pyramid level's model is measured on that level before the denoise.
// measured_raw / measured_pyr (optional) receive the measured models.
template <class T>
inline Plane4<T> raw_pipeline_calibrated(const uint16_t* raw, size_t stride_elems, int w, int h, const Params& p,
                                         float exposure_multiplier, RawNLF* measured_raw = nullptr,
                                         YCbCrNLF* measured_pyr = nullptr) {
    static const Taps t1 = gaussian_bilinear_taps(1.5f), t2 = gaussian_bilinear_taps(4.5f);
    Params q = p;
    q.high_noise = false;
    Plane<T> scaled = scale_raw<T>(raw, stride_elems, w, h, p);
    const Plane4<T> sob = sobel(scaled);
    {
        Plane4<T> mean, var;
        raw_stats(scaled, p.bayer, mean, var);
        q.raw_nlf = measure_raw(mean, var, w, h, exposure_multiplier);
    }
    if (measured_raw) *measured_raw = q.raw_nlf;
    const auto rv = raw_variance(q.raw_nlf);
    const Plane2<T> grad = gradient_blur(scaled, sob, t1, t2, rv[1]);
    Plane4<T> rgb = demosaic(scaled, grad, q.bayer, rv);
    blend_highlights(rgb, T(1));
    const Mat3 c2y = cam_ycbcr(q.rgb_cam, q.xyz_rgb);
    const Mat3 y2c = inverse3(c2y);
    transform(rgb, c2y);
    Plane4<T> ds = despeckle_luma_median_chroma(rgb, p.pyr_nlf[0].a, p.pyr_nlf[0].b);
    {  // the levels as pyramid_denoise builds them, measured before the denoise
        Plane4<T> lvl = ds;
        for (int i = 0; i < q.levels; i++) {
            if (i > 0) lvl = downsample<T, 4>(lvl, w >> i, h >> i, 3);
            q.pyr_nlf[i] = measure_ycc(ycc_stats(lvl), exposure_multiplier);
            if (measured_pyr) measured_pyr[i] = q.pyr_nlf[i];
        }
    }
    Plane4<T> den = pyramid_denoise<T>(ds, grad, q);
    transform(den, y2c);
    return den;
}

}  // namespace nlf
}  // namespace orc
