// gls_calibration.cpp — CameraCalibration<levels> data and schedules
// (MetalPipeline/CameraCalibration.hpp:24-39) for the built-in camera, and
// the host-side parameter helpers the converter needs:
//   * gaussianKernelBilinearWeights (demosaic_utils.cpp:934-1006),
//   * cam_ycbcr (demosaic_utils.cpp:703-720) and its inverse.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "gls_host.h"

namespace gls {

// ---- iPhone 14 Wide noise model (iPhone14WideCalibration.cpp:151-252):
// nine ISO anchors; per anchor the raw NLF (a[4], b[4]) and the per-level
// YCbCr NLF (a[3], b[3]) of a 5-level pyramid. The values are calibration
// data of the reference camera, carried as parameter data.
struct NlfAnchor {
    float raw_a[4], raw_b[4];
    float lvl_a[5][3], lvl_b[5][3];
};

static const NlfAnchor kIphone14Wide[9] = {
    // ISO 50
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {9.605e-05f, 9.510e-05f, 9.561e-05f, 9.557e-05f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{3.021e-05f, 7.708e-06f, 7.702e-06f},
      {8.517e-06f, 6.253e-06f, 5.550e-06f},
      {3.021e-06f, 2.249e-06f, 1.803e-06f},
      {5.619e-06f, 5.195e-07f, 3.991e-07f},
      {1.400e-05f, 2.553e-07f, 8.757e-08f}}},
    // ISO 100
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {2.374e-04f, 2.378e-04f, 2.410e-04f, 2.379e-04f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{3.549e-05f, 1.454e-05f, 1.487e-05f},
      {1.348e-05f, 1.136e-05f, 1.020e-05f},
      {4.445e-06f, 4.221e-06f, 3.552e-06f},
      {7.080e-06f, 1.181e-06f, 8.815e-07f},
      {1.212e-05f, 4.146e-07f, 2.701e-07f}}},
    // ISO 200
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {3.383e-04f, 3.348e-04f, 3.385e-04f, 3.367e-04f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{3.960e-05f, 2.143e-05f, 2.230e-05f},
      {2.195e-05f, 1.877e-05f, 1.727e-05f},
      {6.240e-06f, 7.698e-06f, 6.556e-06f},
      {6.939e-06f, 2.222e-06f, 1.782e-06f},
      {1.201e-05f, 6.308e-07f, 4.537e-07f}}},
    // ISO 400
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {5.231e-04f, 5.169e-04f, 5.199e-04f, 5.173e-04f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{9.127e-05f, 3.411e-05f, 3.599e-05f},
      {3.295e-05f, 2.704e-05f, 2.671e-05f},
      {1.065e-05f, 1.447e-05f, 1.233e-05f},
      {7.496e-06f, 4.304e-06f, 3.577e-06f},
      {1.186e-05f, 1.246e-06f, 9.749e-07f}}},
    // ISO 800
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {1.558e-03f, 1.530e-03f, 1.528e-03f, 1.528e-03f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{1.300e-04f, 6.057e-05f, 6.208e-05f},
      {3.819e-05f, 3.034e-05f, 3.293e-05f},
      {1.778e-05f, 2.436e-05f, 2.191e-05f},
      {9.662e-06f, 8.288e-06f, 6.826e-06f},
      {1.220e-05f, 2.436e-06f, 1.986e-06f}}},
    // ISO 1600
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {2.151e-03f, 2.117e-03f, 2.120e-03f, 2.120e-03f},
     {{1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{2.068e-04f, 1.126e-04f, 1.192e-04f},
      {1.200e-04f, 1.024e-04f, 9.988e-05f},
      {2.003e-05f, 1.876e-05f, 1.880e-05f},
      {1.185e-05f, 1.193e-05f, 1.091e-05f},
      {9.118e-06f, 3.885e-06f, 3.580e-06f}}},
    // ISO 3200
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {7.953e-03f, 7.738e-03f, 7.636e-03f, 7.723e-03f},
     {{6.746e-06f, 2.499e-06f, 2.275e-07f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{3.749e-04f, 1.464e-04f, 1.595e-04f},
      {1.553e-04f, 1.263e-04f, 1.281e-04f},
      {5.782e-05f, 8.328e-05f, 7.481e-05f},
      {1.547e-05f, 1.517e-05f, 1.414e-05f},
      {9.535e-06f, 6.713e-06f, 6.464e-06f}}},
    // ISO 6400
    {{1.000e-08f, 1.000e-08f, 1.000e-08f, 1.000e-08f}, {1.035e-02f, 1.011e-02f, 1.006e-02f, 1.011e-02f},
     {{1.952e-05f, 1.387e-05f, 1.172e-05f}, {1e-8f, 3.489e-06f, 5.335e-06f}, {1e-8f, 3.391e-06f, 3.670e-06f}, {1e-8f, 1e-8f, 1e-8f}, {1e-8f, 1e-8f, 1e-8f}},
     {{1.357e-03f, 5.091e-04f, 5.520e-04f},
      {5.252e-04f, 4.425e-04f, 4.211e-04f},
      {9.430e-05f, 1.116e-04f, 1.068e-04f},
      {3.541e-05f, 4.552e-05f, 4.070e-05f},
      {1.231e-05f, 1.034e-05f, 9.625e-06f}}},
    // ISO 12500
    {{2.052e-03f, 1.942e-03f, 1.908e-03f, 1.944e-03f}, {1.210e-02f, 1.183e-02f, 1.176e-02f, 1.183e-02f},
     {{4.272e-04f, 1.447e-04f, 1.263e-04f},
      {3.231e-05f, 7.428e-05f, 6.601e-05f},
      {1.364e-05f, 2.021e-05f, 2.055e-05f},
      {1.549e-06f, 6.073e-06f, 5.722e-06f},
      {6.605e-07f, 1.290e-06f, 1.209e-06f}},
     {{4.242e-04f, 4.366e-04f, 5.834e-04f},
      {8.655e-04f, 6.859e-04f, 6.985e-04f},
      {1.985e-04f, 3.210e-04f, 3.016e-04f},
      {5.832e-05f, 7.483e-05f, 7.428e-05f},
      {3.724e-05f, 2.416e-05f, 2.349e-05f}}},
};

static float smoothstep_host(float e0, float e1, float x) {  // demosaic.hpp:181-184
    float t = std::clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

static void lerp_anchor(const NlfAnchor& a0, const NlfAnchor& a1, float t, gls_demosaic_params* p) {
    for (int c = 0; c < 4; c++) {
        p->raw_nlf.a[c] = std::lerp(a0.raw_a[c], a1.raw_a[c], t);
        p->raw_nlf.b[c] = std::lerp(a0.raw_b[c], a1.raw_b[c], t);
    }
    for (int l = 0; l < 5; l++)
        for (int c = 0; c < 3; c++) {
            p->pyramid_nlf[l].a[c] = std::lerp(a0.lvl_a[l][c], a1.lvl_a[l][c], t);
            p->pyramid_nlf[l].b[c] = std::lerp(a0.lvl_b[l][c], a1.lvl_b[l][c], t);
        }
}

// iPhone14WideCalibration::nlfFromIso (iPhone14WideCalibration.cpp:33-62).
// The interpolation factor is an integer division, as in the reference, so
// within each ISO bracket it is 0 (the lower anchor) except at the top of
// the last bracket. ISO is clamped to [50, 12500] first.
static void iphone14wide_nlf(int iso, gls_demosaic_params* p) {
    iso = std::clamp(iso, 50, 12500);
    static const int lo[8] = {50, 100, 200, 400, 800, 1600, 3200, 6400};
    int k = 7;
    for (int i = 0; i < 7; i++)
        if (iso >= lo[i] && iso < lo[i + 1]) k = i;
    float a;
    if (k < 7) {
        a = float((iso - lo[k]) / lo[k]);
    } else {
        a = float((iso - 6100) / 6100);
    }
    lerp_anchor(kIphone14Wide[k], kIphone14Wide[k + 1], a, p);
}

// iPhone14WideCalibration::getDenoiseParameters (iPhone14WideCalibration.cpp:65-119).
static void iphone14wide_denoise(int iso, gls_demosaic_params* p) {
    const float highNoiseISO = 100;
    const float nlf_alpha =
        float(std::clamp((std::log2(double(iso)) - std::log2(50.0)) / (std::log2(12500.0) - std::log2(50.0)), 0.0, 1.0));
    const float raw_nlf_alpha = float(std::clamp(
        (std::log2(double(iso)) - std::log2(double(highNoiseISO))) / (std::log2(12500.0) - std::log2(double(highNoiseISO))),
        0.0, 1.0));
    const float lerp = float(std::lerp(1.0, 2.0, double(nlf_alpha)));
    const float lerp_c = 1;
    const float lmult[5] = {3, 1.5f, 1, 1, 1};
    const float cmult[5] = {1, 1, 1, 1, 1};
    for (int l = 0; l < 5; l++) {
        gls_denoise_params& d = p->denoise[l];
        d.luma = lmult[l] * lerp;
        d.chroma = cmult[l] * lerp_c;
        d.chroma_boost = 2;
        d.gradient_boost = 0;
        d.gradient_threshold = 1;
        d.sharpening = 1;
    }
    p->denoise[0].chroma_boost = 8;
    p->denoise[0].gradient_boost = 2 * (2 - smoothstep_host(0.3f, 0.6f, nlf_alpha));
    p->denoise[0].gradient_threshold = 2;
    p->denoise[0].sharpening = std::lerp(1.5f, 1.0f, nlf_alpha);
    p->denoise[1].chroma_boost = 4;
    p->denoise[1].gradient_boost = 2 - smoothstep_host(0.3f, 0.6f, nlf_alpha);
    p->denoise[1].gradient_threshold = 2;
    p->denoise[1].sharpening = 1;
    p->high_noise_image = iso >= highNoiseISO ? 1 : 0;
    p->raw_denoise_strength = std::lerp(0.5f, 3.0f, raw_nlf_alpha);
    p->iso = iso;
}

gls_status calibration_fill(int camera, int iso, gls_demosaic_params* p) {
    if (!p) return set_error(GLS_ERR_INVALID_ARG, "gls_calibration_fill: params is NULL");
    if (camera != GLS_CAMERA_IPHONE14_WIDE)
        return set_error(GLS_ERR_INVALID_ARG, "gls_calibration_fill: unknown camera id");
    if (iso <= 0) return set_error(GLS_ERR_RANGE, "gls_calibration_fill: ISO must be positive");
    iphone14wide_nlf(iso, p);
    iphone14wide_denoise(iso, p);
    // buildDemosaicParameters, iPhone14WideCalibration.cpp:121-137
    p->lens_shading_correction = 1.6f;
    p->rgb_conversion.contrast = 1.05f;
    p->rgb_conversion.saturation = 1.0f;
    p->rgb_conversion.tone_curve_slope = 3.5f;
    p->rgb_conversion.exposure_bias = 0.0f;
    p->rgb_conversion.blacks = 0.0f;
    p->rgb_conversion.local_tone_mapping = 1;
    p->ltm.eps = 0.01f;
    p->ltm.shadows = 1.0f;
    p->ltm.highlights = 1.0f;
    p->ltm.detail[0] = 1.0f;
    p->ltm.detail[1] = 1.5f;
    p->ltm.detail[2] = 2.0f;
    if (p->levels <= 0) p->levels = 5;
    return GLS_OK;
}

// gaussianKernelBilinearWeights + KernelOptimizeBilinear2d,
// demosaic_utils.cpp:934-1006: a (2k+1)^2 Gaussian folded into (k+1)^2
// bilinear taps (weight, dx, dy). The last tap's offsets are width/2.0f as
// in the reference (demosaic_utils.cpp:984).
int gaussian_taps(float radius, float* out, int max_taps) {
    int ks = std::max(int(std::ceil(2 * radius)), 2);
    if ((ks % 2) == 0) ks++;
    const int ow = ks / 2 + 1, half = ks / 2;
    const int n = ow * ow;
    if (n > max_taps) return -n;
    float w[64 * 64];
    if (ks > 64) return -n;
    for (int y = -half, i = 0; y <= half; y++)
        for (int x = -half; x <= half; x++, i++)
            w[i] = float(std::exp(-(double(float(x * x + y * y)) / double(2 * radius * radius))));
    auto put = [&](int k, float a, float b, float c) {
        out[3 * k] = a;
        out[3 * k + 1] = b;
        out[3 * k + 2] = c;
    };
    int row, col;
    for (row = 0; row < ks - 1; row += 2) {
        for (col = 0; col < ks - 1; col += 2) {
            const float w1 = w[row * ks + col], w2 = w[row * ks + col + 1];
            const float w3 = w[(row + 1) * ks + col], w4 = w[(row + 1) * ks + col + 1];
            const float x1 = float(col - half), x2 = float(col - half + 1);
            const float y1 = float(row - half), y2 = float(row - half + 1);
            put((row / 2) * ow + col / 2, w1 + w2 + w3 + w4, (x1 * w1 + x2 * w2) / (w1 + w2), (y1 * w1 + y2 * w3) / (w1 + w3));
        }
        const float w1 = w[row * ks + col], w2 = w[(row + 1) * ks + col];
        const float y1 = float(row - half), y2 = float(row - half + 1);
        put((row / 2) * ow + col / 2, w1 + w2, float(col - half), (y1 * w1 + y2 * w2) / (w1 + w2));
    }
    for (col = 0; col < ks - 1; col += 2) {
        const float w1 = w[row * ks + col], w2 = w[row * ks + col + 1];
        const float x1 = float(col - half), x2 = float(col - half + 1);
        put((row / 2) * ow + col / 2, w1 + w2, (x1 * w1 + x2 * w2) / (w1 + w2), float(row - half));
    }
    put((row / 2) * ow + col / 2, w[row * ks + col], ks / 2.0f, ks / 2.0f);
    return n;
}

// cam_ycbcr, demosaic_utils.cpp:703-720, and its inverse (computed in
// double, rounded to float).
void cam_ycbcr(const float rgb_cam[9], const float xyz_rgb[9], float fwd[9], float inv[9]) {
    float cam_y[3];
    for (int j = 0; j < 3; j++)
        cam_y[j] = xyz_rgb[3] * rgb_cam[j] + xyz_rgb[4] * rgb_cam[3 + j] + xyz_rgb[5] * rgb_cam[6 + j];
    const float KR = cam_y[0], KG = cam_y[1], KB = cam_y[2];
    const float m[9] = {KR, KG, KB,
                        -0.5f * KR / (1.0f - KB), -0.5f * KG / (1 - KB), 0.5f,
                        0.5f, -0.5f * KG / (1 - KR), -0.5f * KB / (1 - KR)};
    std::memcpy(fwd, m, sizeof(m));
    double a[3][3];
    for (int i = 0; i < 9; i++) a[i / 3][i % 3] = m[i];
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    const double r[9] = {c00, a[0][2] * a[2][1] - a[0][1] * a[2][2], a[0][1] * a[1][2] - a[0][2] * a[1][1],
                         c01, a[0][0] * a[2][2] - a[0][2] * a[2][0], a[0][2] * a[1][0] - a[0][0] * a[1][2],
                         c02, a[0][1] * a[2][0] - a[0][0] * a[2][1], a[0][0] * a[1][1] - a[0][1] * a[1][0]};
    for (int i = 0; i < 9; i++) inv[i] = float(r[i] / det);
}

}  // namespace gls
