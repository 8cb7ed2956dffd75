// gls_oracle_post.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the
// reference's display post-processing (RawConverter::demosaic with
// postProcess, raw_converter.cpp:80-116, 224-244): the histogram of the
// denoised level 3 and its statistics, the three-band local tone mapping
// mask (guided filter on denoised levels 4, 2 and 0) and convertTosRGB
// with its Perlin grain. The checker for the CUDA post-processing; nothing
// in the product links it.
//
// Semantics fixed here and in the CUDA kernels alike (the reference leaves
// them to Apple's texture unit):
//   * the guided filter's 5x5 samples and the box filter's 9 taps are read
//     at their texel positions (x + dx, y + dy), clamp-to-edge; the
//     reference forms them as normalised coordinates that the hardware
//     turns back into texel positions with its own rounding;
//   * the mask reads each band's (a, b) plane bilinearly at
//     (x + 0.5) * (band width / width) - 0.5, the convention of the
//     pyramid's up-sampling.
// The statistics are float, one thread, in the reference's order, so the
// integer histogram and its thresholds are exact.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "gls_oracle.hpp"

namespace orc {
namespace post {

struct PostParams {
    float contrast = 1.05f, saturation = 1.0f, slope = 3.5f, bias = 0.0f, blacks = 0.0f;
    bool ltm = false;
    float eps = 0.01f, detail[3] = {1, 1, 1};
    float nlf[2] = {0, 0};         // pyramid_nlf[0] luma (a, b): the high band's noise gate
    float luma_var[2] = {0, 0};    // 2 x the raw green variance (a, b): the grain's sigma
    float rgb_cam[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
};

// histogram_data (demosaic.metal:1360-1369) after histogramStatistics
struct Stats {
    uint32_t hist[256] = {};
    uint32_t bands[8] = {};
    float black = 0, white = 0, shadows = 0, highlights = 0, mean = 0, median = 0;
};

inline float smooth_f(float e0, float e1, float x) { return smoothstepT<float>(e0, e1, x); }

// histogramImage + histogramStatistics (demosaic.metal:1373-1455) over the
// luma of the denoised level image
template <class T>
inline Stats histogram(const Plane4<T>& img) {
    Stats s;
    for (int y = 0; y < img.h; y++)
        for (int x = 0; x < img.w; x++) {
            const float v = float(img.px(x, y)[0]);
            const int idx = std::clamp(int(255.0f * std::sqrt(v / 2.0f)), 0, 255);
            s.hist[idx]++;
        }
    const uint32_t image_size = uint32_t(img.w) * uint32_t(img.h);
    float mean = 0;
    bool found_median = false, found_black = false, found_white = false;
    int median_index = 0, black_index = 0, white_index = 0;
    uint32_t sum = 0;
    for (int band = 0; band < 8; band++)
        for (int i = 0; i < 32; i++) {
            const int index = band * 32 + i;
            const uint32_t entry = s.hist[index];
            s.bands[band] += entry;
            mean += float(entry * uint32_t(index + 1)) / 256.0f;
            sum += entry;
            if (!found_median && sum >= (image_size + 1) / 2) {
                median_index = index;
                found_median = true;
            }
            if (!found_black && float(sum) >= 0.001f * float(image_size)) {
                black_index = index;
                found_black = true;
            }
            if (!found_white && float(sum) >= 0.999f * float(image_size)) {
                white_index = index;
                found_white = true;
            }
        }
    mean /= float(image_size);
    {
        const float v = float(black_index - 1) / 255.0f;
        s.black = 2.0f * v * v;
    }
    {
        const float v = float(white_index) / 255.0f;
        s.white = 2.0f * v * v;
    }
    s.median = float(median_index) / 255.0f - s.black;
    s.mean = mean - s.black;
    s.highlights = 1.0f + 2.0f * smooth_f(0.01f, 0.1f, float(s.bands[5] + s.bands[6] + s.bands[7]) / float(image_size));
    s.shadows = 0.8f - 0.5f * smooth_f(0.25f, 0.5f, float(s.bands[0] + s.bands[1]) / float(image_size));
    return s;
}

// without noise reduction the reference sets fixed levels on the zeroed
// histogram data (raw_converter.cpp:224-229)
inline Stats fixed_stats() {
    Stats s;
    s.black = 0.1f;
    s.white = 1.0f;
    s.mean = 0.22f;
    s.median = 0.22f;
    return s;
}

// Noise2D::randomSeed + initGradients (SimplexNoise.hpp:109-143), B = 256,
// from the C library's srandom / random
struct NoiseTables {
    int perm[514];
    float grad[514][2];
};

inline NoiseTables noise_tables(unsigned seed) {
    NoiseTables t;
    srandom(seed);
    for (int i = 0; i < 256; i++) {
        t.perm[i] = i;
        for (int j = 0; j < 2; j++) t.grad[i][j] = float((random() % 512) - 256) / 256;
        const float s = std::sqrt(t.grad[i][0] * t.grad[i][0] + t.grad[i][1] * t.grad[i][1]);
        t.grad[i][0] = t.grad[i][0] / s;
        t.grad[i][1] = t.grad[i][1] / s;
    }
    for (int i = 255; i > 0; i--) {
        const int k = t.perm[i];
        const int j = int(random() % 256);
        t.perm[i] = t.perm[j];
        t.perm[j] = k;
    }
    for (int i = 0; i < 258; i++) {
        t.perm[256 + i] = t.perm[i];
        t.grad[256 + i][0] = t.grad[i][0];
        t.grad[256 + i][1] = t.grad[i][1];
    }
    return t;
}

// noise / octaveNoise (demosaic.metal:1558-1602), float as in Metal
inline float noise(const NoiseTables& T_, float px, float py) {
    const float tx = px + 4096.0f, ty = py + 4096.0f;
    const int b0x = int(tx) & 255, b0y = int(ty) & 255;
    const int b1x = (b0x + 1) & 255, b1y = (b0y + 1) & 255;
    const float r0x = tx - std::floor(tx), r0y = ty - std::floor(ty);
    const float r1x = r0x - 1, r1y = r0y - 1;
    const int i = T_.perm[b0x], j = T_.perm[b1x];
    const int b00 = T_.perm[i + b0y], b10 = T_.perm[j + b0y], b01 = T_.perm[i + b1y], b11 = T_.perm[j + b1y];
    const float sx = r0x * r0x * (3.0f - 2.0f * r0x), sy = r0y * r0y * (3.0f - 2.0f * r0y);
    auto dot2 = [&](int g, float ax, float ay) { return T_.grad[g][0] * ax + T_.grad[g][1] * ay; };
    float u = dot2(b00, r0x, r0y), v = dot2(b10, r1x, r0y);
    const float a = u + (v - u) * sx;
    u = dot2(b01, r0x, r1y);
    v = dot2(b11, r1x, r1y);
    const float b = u + (v - u) * sx;
    return a + (b - a) * sy;
}

inline float octave_noise(const NoiseTables& t, float px, float py) {
    float freq = 1.0f, amp = 1.0f, norm = 1.0f;
    float sum = noise(t, px, py);
    for (int i = 1; i < 4; ++i) {
        freq *= 0.5f;
        amp *= 0.5f;
        norm += amp;
        sum += noise(t, px * freq, py * freq) * amp;
    }
    return sum / norm;
}

// GuidedFilterABImage (demosaic.metal:1295-1321): (a, b) of a 5x5 window of
// the guide's luma
template <class T>
inline Plane2<T> guided_ab(const Plane4<T>& g, float eps) {
    Plane2<T> ab(g.w, g.h);
    parallel_rows(g.h, [&](int y) {
        for (int x = 0; x < g.w; x++) {
            T sum = 0, sumSq = 0;
            for (int dy = -2; dy <= 2; dy++)
                for (int dx = -2; dx <= 2; dx++) {
                    const T s = g.at(x + dx, y + dy, 0);
                    sum += s;
                    sumSq += s * s;
                }
            const T mean = sum / T(25);
            const T var = (sumSq - sum * sum / T(25)) / T(25);
            const T a = var / (var + T(eps));
            ab.px(x, y)[0] = a;
            ab.px(x, y)[1] = mean * (T(1) - a);
        }
    });
    return ab;
}

// BoxFilterGFImage (demosaic.metal:1323-1356): a 5x5 box as nine bilinear
// taps at half-texel offsets
template <class T>
inline Plane2<T> box_ab(const Plane2<T>& in) {
    static const float w[9] = {0.16f, 0.16f, 0.08f, 0.16f, 0.16f, 0.08f, 0.08f, 0.08f, 0.04f};
    static const float ox[9] = {-1.5f, 0.5f, 2.0f, -1.5f, 0.5f, 2.0f, -1.5f, 0.5f, 2.0f};
    static const float oy[9] = {-1.5f, -1.5f, -1.5f, 0.5f, 0.5f, 0.5f, 2.0f, 2.0f, 2.0f};
    Plane2<T> out(in.w, in.h);
    parallel_rows(in.h, [&](int y) {
        for (int x = 0; x < in.w; x++)
            for (int c = 0; c < 2; c++) {
                T m = 0;
                for (int i = 0; i < 9; i++) m += T(w[i]) * in.bilin(T(x) + T(ox[i]), T(y) + T(oy[i]), c);
                out.px(x, y)[c] = m;
            }
    });
    return out;
}

// computeLtmMultiplier (demosaic.metal:1457-1472)
template <class T>
inline T ltm_multiplier(T Y, T ill, T shadows, T highlights, T detail) {
    const T mid = T(0.22f);
    const T refl = Y / ill;
    const T adj = ill <= mid ? mid * std::pow(ill / mid, shadows)
                             : (T(1) - mid) * std::pow((ill - mid) / (T(1) - mid), highlights) + mid;
    return adj * std::pow(refl, detail) / Y;
}

// localToneMappingMaskImage (demosaic.metal:1481-1544) at one pixel
template <class T>
inline T ltm_mask(const Plane4<T>& den0, const Plane2<T>& grad, const Plane2<T>* ab[3], const PostParams& pp,
                  const Stats& st, int x, int y) {
    const T Y = den0.px(x, y)[0];
    T mult = 1;
    for (int k = 0; k < 3; k++) {
        const Plane2<T>& m = *ab[k];
        const T u = (T(x) + T(0.5)) * (T(m.w) / T(den0.w)) - T(0.5);
        const T v = (T(y) + T(0.5)) * (T(m.h) / T(den0.h)) - T(0.5);
        const T ill = m.bilin(u, v, 0) * Y + m.bilin(u, v, 1);
        T d = pp.detail[k];
        if (d > T(1)) {
            T dd = (T(1) - smoothstepT<T>(T(0.75), T(0.95), ill)) * smoothstepT<T>(T(0.05), T(0.1), ill);
            if (k == 2) {
                const T gx = grad.px(x, y)[0], gy = grad.px(x, y)[1];
                const T g = std::sqrt(gx * gx + gy * gy);
                const T sigma = std::sqrt(T(pp.nlf[0]) + T(pp.nlf[1]) * ill);
                dd = smoothstepT<T>(T(2) * sigma, T(8) * sigma, g) *
                     (T(1) - smoothstepT<T>(T(32) * sigma, T(128) * sigma, g)) * dd;
            }
            d = T(1) + (d - T(1)) * dd;
        }
        mult *= ltm_multiplier<T>(Y, ill, T(st.shadows), k == 0 ? T(st.highlights) : T(1), d);
    }
    return mult;
}

template <class T>
inline T sigmoid(T x, T s) {
    return T(0.5) * (std::tanh(s * x - T(0.3) * s) + T(1));
}
// toneCurve (demosaic.metal:600-609)
template <class T>
inline T tone_curve(T x, T s) {
    return (sigmoid<T>(std::pow(T(0.95) * x, T(0.5)), s) - sigmoid<T>(T(0), s)) /
           (sigmoid<T>(T(1), s) - sigmoid<T>(T(0), s));
}

// convertTosRGB (demosaic.metal:1621-1705) at one pixel; rgb_in is the
// linear camera RGB, mask the LTM boost (used when pp.ltm)
template <class T>
inline void to_srgb(const T rgb_in[3], T mask, const PostParams& pp, const Stats& st, const NoiseTables& nt, int x,
                    int y, T out[4]) {
    const T black = T(st.black), white = T(1);
    T brightening = 1;
    if (T(st.mean) > T(0.22)) brightening *= T(0.22) / T(st.mean);
    T pv[3];
    for (int c = 0; c < 3; c++) pv[c] = brightening * std::max(rgb_in[c] - black, T(0)) / (white - black);
    if (pp.bias != 0) {
        const T e = std::pow(T(2), T(pp.bias));
        for (int c = 0; c < 3; c++) pv[c] *= e;
    }
    if (pp.saturation != 1.0f) {
        const T luma = T(0.2126) * pv[0] + T(0.7152) * pv[1] + T(0.0722) * pv[2];
        for (int c = 0; c < 3; c++)
            pv[c] = mixT<T>(luma, pv[c], mixT<T>(T(pp.saturation), T(1), smoothstepT<T>(T(0.75), T(2), pv[c])));
    }
    if (pp.contrast != 1.0f) {
        for (int c = 0; c < 3; c++)
            pv[c] = mixT<T>(T(0.2), pv[c], mixT<T>(T(pp.contrast), T(1), smoothstepT<T>(T(0.9), T(2), pv[c])));
    }
    T rgb[3];
    for (int c = 0; c < 3; c++)
        rgb[c] = std::max(T(pp.rgb_cam[3 * c]) * pv[0] + T(pp.rgb_cam[3 * c + 1]) * pv[1] +
                              T(pp.rgb_cam[3 * c + 2]) * pv[2],
                          T(0));
    T sigma = 0;
    const bool lv = pp.luma_var[0] != 0 || pp.luma_var[1] != 0;
    if (pp.ltm) {
        const T boost = mask;
        if (boost > T(1)) {
            const T luma = T(0.2126) * rgb[0] + T(0.7152) * rgb[1] + T(0.0722) * rgb[2];
            const T t = std::min(std::pow(luma, T(0.5)), T(1));
            const T s = smoothstepT<T>(T(0.5), T(0.8), luma);
            for (int c = 0; c < 3; c++) {
                const T lifted = T(1) - (T(1) - rgb[c]) * (T(1) - boost * luma) / (T(1) - luma);
                rgb[c] = mixT<T>(rgb[c] * boost, mixT<T>(lifted, rgb[c] * boost, s), t);
            }
        } else if (boost < T(1)) {
            for (int c = 0; c < 3; c++) rgb[c] *= boost;
        }
        if (lv) sigma = std::sqrt(T(pp.luma_var[0]) + T(pp.luma_var[1]) * boost * rgb_in[1]);
    } else if (lv) {
        sigma = std::sqrt(T(pp.luma_var[0]) + T(pp.luma_var[1]) * rgb_in[1]);
    }
    if (sigma > T(0)) {
        const T n = T(octave_noise(nt, 0.5f * float(x), 0.5f * float(y)));
        for (int c = 0; c < 3; c++) rgb[c] += sigma * n;
    }
    for (int c = 0; c < 3; c++) {
        T v = tone_curve<T>(std::max(rgb[c], T(0)), T(pp.slope));
        if (pp.blacks > 0) v = (v - T(pp.blacks)) / (T(1) - T(pp.blacks));
        out[c] = clampT<T>(v, T(0), T(1));
    }
    out[3] = T(1);
}

// The post-processing of one frame: den = the denoised levels (YCbCr,
// 5 levels, or empty without noise reduction), rgb = the linear camera RGB
// output, grad the level-0 gradient plane; seed = the raw frame's first
// pixel (raw_converter.cpp:238).
template <class T>
inline Plane4<T> postprocess(const std::vector<Plane4<T>>& den, const Plane2<T>& grad, const Plane4<T>& rgb,
                             const PostParams& pp, unsigned seed, Stats* stats_out = nullptr) {
    const bool denoise = den.size() == 5;
    const Stats st = denoise ? histogram(den[3]) : fixed_stats();
    if (stats_out) *stats_out = st;
    const NoiseTables nt = noise_tables(seed);
    std::vector<Plane2<T>> ab;
    const bool ltm = pp.ltm && denoise;
    if (ltm)
        for (int k : {4, 2, 0}) ab.push_back(box_ab(guided_ab(den[k], pp.eps)));
    PostParams p2 = pp;
    p2.ltm = ltm;
    Plane4<T> out(rgb.w, rgb.h);
    parallel_rows(rgb.h, [&](int y) {
        for (int x = 0; x < rgb.w; x++) {
            T mask = 1;
            if (ltm) {
                const Plane2<T>* bands[3] = {&ab[0], &ab[1], &ab[2]};
                mask = ltm_mask<T>(den[0], grad, bands, p2, st, x, y);
            }
            to_srgb<T>(rgb.px(x, y), mask, p2, st, nt, x, y, out.px(x, y));
        }
    });
    return out;
}

}  // namespace post
}  // namespace orc
