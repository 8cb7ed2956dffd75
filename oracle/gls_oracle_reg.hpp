// gls_oracle_reg.hpp — TEST INFRASTRUCTURE ONLY. CPU restatement of the
// registration and fusion rows of the GlassCamera path: RawChannels and its
// tone curve, the SURF integral image, fast-Hessian detector, orientation
// and 64-D descriptor, brute-force matching, RANSAC + least-squares
// homography, and the registerAndFuse / registerImage / registerBayerImage
// warps. Nothing in the product links or calls this code.
//
// Each function cites the reference file:line it restates (paths relative to
// the GlassCameraPublic tree). The reference splits this work between Metal
// kernels (ImageRegistration/SURF.metal) and C++ (ImageRegistration/SURF.cpp,
// Homography.cpp, LeastSquaresHomography.cpp, RTL/RANSAC.hpp,
// PyramidFusion/pyramidFusion.cpp); each piece follows the variant the
// reference's live path runs (USE_GPU_HESSIAN_DETECTOR, USE_GPU_KEYPOINT_MATCH,
// USE_RTL are true; USE_INTEGRAL_PYRAMID is false; SURF.cpp:31-34,
// Homography.cpp:22-23).
//
// Semantics fixed here and in the CUDA kernels alike:
//   * every float expression is evaluated as written, one rounding per
//     operation, no FMA contraction (the Metal kernels build with fast math,
//     whose contraction choices are not specified);
//   * atan2f / sinf / cosf are the library's own (gls_fmath.h), so the two
//     sides agree to the bit; they stay within a few ulps of libm;
//   * hypot in the Jacobi solver is sqrt(p^2 + y^2) in double;
//   * registerAndFuse samples the input by exact bilinear interpolation at
//     texel position (x', y') = H (x, y) with clamp-to-edge, the texel-space
//     reading of the reference's (x' + 0.5) / size normalised coordinate;
//   * RANSAC draws its 4-point samples from std::mt19937 (default seed, as
//     the reference's default-constructed engine) through a uniform integer
//     map given by the caller: the product uses mask-and-reject over the
//     engine's low bits (the algorithm of the LLVM C++ library the reference
//     builds with); the pin against the reference compiled here uses this
//     toolchain's std::uniform_int_distribution, as that build does.
#pragma once

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <random>
#include <set>
#include <vector>

#include "../glasscamerapublic_b200/csrc/gls_fmath.h"
#include "gls_oracle.hpp"

namespace orc {
namespace reg {

using glsm::fadd;
using glsm::fdiv;
using glsm::fmul;
using glsm::fsub;

// ------------------------------------------------------------ plain images
struct FImg {
    int w = 0, h = 0;
    std::vector<float> d;
    FImg() = default;
    FImg(int w_, int h_) : w(w_), h(h_), d(size_t(w_) * h_, 0.0f) {}
    float& at(int x, int y) { return d[size_t(y) * w + x]; }
    float at(int x, int y) const { return d[size_t(y) * w + x]; }
};

// ------------------------------------------------------------ RawChannels
// sigmoid / toneCurve (PyramidFusion/pyramidFusion.cpp:92-104), evaluated
// with the reference's mix of float and double.
inline float sigmoid(float x, float s) { return float(0.5 * (std::tanh(double(s * x) - 0.3 * s) + 1)); }

inline float tone_curve(float x, float s) {
    const float p = float(std::pow(0.95 * x, 0.5));
    return (sigmoid(p, s) - sigmoid(0.0f, s)) / (sigmoid(1.0f, s) - sigmoid(0.0f, s));
}

// Host Bayer table (MetalPipeline/demosaic.hpp:128-133): per pattern the
// (x, y) offsets of channels R, G, B, G2.
static const int kHostBayer[4][4][2] = {
    {{1, 0}, {0, 0}, {0, 1}, {1, 1}},  // grbg
    {{0, 1}, {0, 0}, {1, 0}, {1, 1}},  // gbrg
    {{0, 0}, {1, 0}, {1, 1}, {0, 1}},  // rggb
    {{1, 1}, {1, 0}, {0, 0}, {0, 1}},  // bggr
};

// RawChannels (pyramidFusion.cpp:106-143): channel c of the quad at half
// resolution through the tone curve at strength 3.5.
inline FImg raw_channel(const uint16_t* raw, int w, int h, size_t stride_px, int pattern, int c, float black,
                        float white, float exposure) {
    FImg out(w / 2, h / 2);
    const int ox = kHostBayer[pattern][c][0], oy = kHostBayer[pattern][c][1];
    for (int y = 0; y < out.h; y++)
        for (int x = 0; x < out.w; x++) {
            const float v = float(raw[size_t(2 * y + oy) * stride_px + 2 * x + ox]);
            const float a = exposure * (v - black) / white;
            out.at(x, y) = tone_curve(std::clamp(a, 0.0f, 1.0f), 3.5f);
        }
    return out;
}

// ------------------------------------------------------------ integral image
// integral_sum_cols_image + integral_sum_rows_image (SURF.metal:315-421),
// driven by integralImageKernel (SURF.cpp:776-825): a per-column running
// sum of (v - 0.5) down the rows, then a per-row running sum of those along
// the columns, both sequential in float. Output (W+1) x (H+1) with a zero
// first row and column.
inline FImg integral(const FImg& img) {
    FImg col(img.w, img.h), sum(img.w + 1, img.h + 1);
    for (int x = 0; x < img.w; x++) {
        float acc = 0.0f;
        for (int y = 0; y < img.h; y++) {
            acc = fadd(acc, fsub(img.at(x, y), 0.5f));
            col.at(x, y) = acc;
        }
    }
    for (int y = 0; y < img.h; y++) {
        float acc = 0.0f;
        for (int x = 0; x < img.w; x++) {
            acc = fadd(acc, col.at(x, y));
            sum.at(x + 1, y + 1) = acc;
        }
    }
    return sum;
}

// ------------------------------------------------------------ Haar patterns
struct HaarBox {
    int x1, y1, x2, y2;
    float w;
};

// resizeHaarPattern (SURF.cpp:103-114)
template <size_t N>
std::array<HaarBox, N> resize_haar(const int src[N][5], int old_size, int new_size) {
    std::array<HaarBox, N> dst;
    const float ratio = float(new_size) / float(old_size);
    for (size_t k = 0; k < N; k++) {
        const int dx1 = int(std::lrint(ratio * float(src[k][0])));
        const int dy1 = int(std::lrint(ratio * float(src[k][1])));
        const int dx2 = int(std::lrint(ratio * float(src[k][2])));
        const int dy2 = int(std::lrint(ratio * float(src[k][3])));
        dst[k] = {dx1, dy1, dx2, dy2, float(src[k][4]) / (float(dx2 - dx1) * float(dy2 - dy1))};
    }
    return dst;
}

// DetAndTraceHaarPattern (SURF.cpp:227-305): the 9x9 box-filter Hessian
// patterns scaled to `size`, and the margin crop of valid sample positions.
struct LayerPattern {
    std::array<HaarBox, 3> dx, dy;
    std::array<HaarBox, 4> dxy;
    int mx, my, mw, mh;  // margin crop (in layer samples)
};

inline LayerPattern layer_pattern(int sum_w, int sum_h, int size, int step) {
    static const int dx_s[3][5] = {{0, 2, 3, 7, 1}, {3, 2, 6, 7, -2}, {6, 2, 9, 7, 1}};
    static const int dy_s[3][5] = {{2, 0, 7, 3, 1}, {2, 3, 7, 6, -2}, {2, 6, 7, 9, 1}};
    static const int dxy_s[4][5] = {{1, 1, 4, 4, 1}, {5, 1, 8, 4, -1}, {1, 5, 4, 8, -1}, {5, 5, 8, 8, 1}};
    LayerPattern L;
    L.dx = resize_haar<3>(dx_s, 9, size);
    L.dy = resize_haar<3>(dy_s, 9, size);
    L.dxy = resize_haar<4>(dxy_s, 9, size);
    L.mx = (size / 2) / step;
    L.my = (size / 2) / step;
    L.mw = 1 + (sum_w - 1 - size) / step;
    L.mh = 1 + (sum_h - 1 - size) / step;
    if (size > sum_w - 1 || size > sum_h - 1) L.mw = L.mh = 0;  // the wavelet does not fit: no samples
    return L;
}

// integralRectangle of the Metal kernels (SURF.metal:68-71): float 0.5.
inline float rect_gpu(float tr, float tl, float br, float bl) { return fsub(fadd(0.5f, fsub(tr, tl)), fsub(br, bl)); }

// calcHaarPatternDx / Dy / Dxy (SURF.metal:77-125) with the offsets that
// gpuSurfHF (SURF.cpp:200-225) packs: Dx reads the corners of the outer box
// (boxes 0 and 2 share rows) and of the middle box, weighted +w and -3w.
inline float haar_dx(const FImg& s, int px, int py, const LayerPattern& L) {
    const HaarBox &b0 = L.dx[0], &b1 = L.dx[1], &b2 = L.dx[2];
    auto S = [&](int x, int y) { return s.at(px + x, py + y); };
    const float r02 = S(b0.x1, b0.y1), r07 = S(b0.x1, b0.y2), r32 = S(b0.x2, b0.y1), r37 = S(b0.x2, b0.y2);
    const float r62 = S(b1.x2, b1.y1), r67 = S(b1.x2, b1.y2);
    const float r92 = S(b2.x2, b2.y1), r97 = S(b2.x2, b2.y2);
    const float w = L.dx[0].w;
    return fmul(w, fsub(rect_gpu(r97, r92, r07, r02), fmul(3.0f, rect_gpu(r67, r62, r37, r32))));
}

inline float haar_dy(const FImg& s, int px, int py, const LayerPattern& L) {
    const HaarBox &b0 = L.dy[0], &b1 = L.dy[1], &b2 = L.dy[2];
    auto S = [&](int x, int y) { return s.at(px + x, py + y); };
    // p_dy[0] = corners of box 0: (x1,y1) (x1,y2) (x2,y1) (x2,y2)
    const float r20 = S(b0.x1, b0.y1), r23 = S(b0.x1, b0.y2), r70 = S(b0.x2, b0.y1), r73 = S(b0.x2, b0.y2);
    // p_dy[1] = (x1,y2) (x2,y2) of boxes 1 and 2
    const float r26 = S(b1.x1, b1.y2), r76 = S(b1.x2, b1.y2);
    const float r29 = S(b2.x1, b2.y2), r79 = S(b2.x2, b2.y2);
    const float w = L.dx[0].w;
    return fmul(w, fsub(rect_gpu(r79, r70, r29, r20), fmul(3.0f, rect_gpu(r76, r73, r26, r23))));
}

inline float haar_dxy(const FImg& s, int px, int py, const LayerPattern& L) {
    const float w = L.dxy[0].w;
    const float w4[4] = {w, -w, -w, w};
    float d = 0.0f;
    for (int k = 0; k < 4; k++) {
        const HaarBox& b = L.dxy[k];
        const float p0 = s.at(px + b.x1, py + b.y1), p1 = s.at(px + b.x1, py + b.y2);
        const float p2 = s.at(px + b.x2, py + b.y1), p3 = s.at(px + b.x2, py + b.y2);
        d = fadd(d, fmul(w4[k], rect_gpu(p0, p1, p2, p3)));
    }
    return d;
}

// calcDetAndTrace (SURF.metal:127-145)
inline void det_trace(const FImg& sum, int px, int py, const LayerPattern& L, float* det, float* trace) {
    const float dx = haar_dx(sum, px, py, L);
    const float dy = haar_dy(sum, px, py, L);
    const float dxy = haar_dxy(sum, px, py, L);
    *det = fsub(fmul(dx, dy), fmul(fmul(0.81f, dxy), dxy));
    *trace = fadd(dx, dy);
}

// ------------------------------------------------------------ keypoints
struct KeyPoint {  // feature2d.hpp:25-47 (28 bytes)
    float x, y, size, angle, response;
    int octave, class_id;
};

// KeypointGreater (SURF.cpp:1215-1227)
inline bool keypoint_greater(const KeyPoint& a, const KeyPoint& b) {
    if (a.response > b.response) return true;
    if (a.response < b.response) return false;
    if (a.size > b.size) return true;
    if (a.size < b.size) return false;
    if (a.octave > b.octave) return true;
    if (a.octave < b.octave) return false;
    if (a.y < b.y) return false;
    if (a.y > b.y) return true;
    return a.x < b.x;
}

inline float det3(const float a[3], const float b[3], const float c[3]) {
    // dot(A0, cross(A1, A2)) (SURF.metal:184-187)
    const float cx = fsub(fmul(b[1], c[2]), fmul(b[2], c[1]));
    const float cy = fsub(fmul(b[2], c[0]), fmul(b[0], c[2]));
    const float cz = fsub(fmul(b[0], c[1]), fmul(b[1], c[0]));
    return fadd(fadd(fmul(a[0], cx), fmul(a[1], cy)), fmul(a[2], cz));
}

struct SurfConfig {
    int n_octaves = 4, n_octave_layers = 2;
    float hessian_threshold = 0.02f;
    int max_features = 1500;
    // false: the reference's detector. Its interpolation step
    // (SURF.metal:200) returns `(float3)(a, b, c) / det`, which C++ (and
    // Metal, a C++14 dialect) reads as a cast of the comma expression:
    // float3(c) / det, the scale offset in all three lanes; and it describes
    // only some keypoints of a small set (described_keypoints). true: the
    // corrected detector, per-axis Cramer solve and every keypoint described.
    bool per_axis_interp = false;
};

// fastHessianDetector (SURF.cpp:1229-1286) with calcDetAndTrace and
// findMaximaInLayer (SURF.metal:127-145, 249-313) and interpolateKeypoint
// (SURF.metal:207-247); det planes outside each layer's margin crop are
// zero. Returns the keypoints sorted by KeypointGreater, all of them (the
// max_features cut is the caller's, SURF.cpp:1413-1418).
inline std::vector<KeyPoint> detect(const FImg& sum, int width, int height, const SurfConfig& cfg) {
    const int layers = cfg.n_octave_layers + 2;
    const int total = layers * cfg.n_octaves;
    std::vector<int> sizes(total), steps(total);
    std::vector<FImg> dets(total);
    for (int o = 0, idx = 0; o < cfg.n_octaves; o++)
        for (int l = 0; l < layers; l++, idx++) {
            sizes[idx] = (9 + 6 * l) << o;
            steps[idx] = 1 << o;
        }
    parallel_rows(total, [&](int i) {
        const int step = steps[i];
        FImg det(width / step, height / step);
        const LayerPattern L = layer_pattern(sum.w, sum.h, sizes[i], step);
        for (int y = 0; y < L.mh; y++)
            for (int x = 0; x < L.mw; x++) {
                float d, t;
                det_trace(sum, x * step, y * step, L, &d, &t);
                det.at(x + L.mx, y + L.my) = d;
            }
        dets[i] = std::move(det);
    });
    std::vector<KeyPoint> kps;
    for (int o = 0; o < cfg.n_octaves; o++)
        for (int l = 1; l <= cfg.n_octave_layers; l++) {
            const int layer = o * layers + l;
            const int step = steps[layer];
            const int s0 = sizes[layer - 1], size = sizes[layer], s2 = sizes[layer + 1];
            const int lw = width / step, lh = height / step;
            const int margin = (s2 / 2) / step + 1;
            const FImg &D0 = dets[layer - 1], &D1 = dets[layer], &D2 = dets[layer + 1];
            const LayerPattern L = layer_pattern(sum.w, sum.h, size, step);
            for (int y = margin; y < lh - margin; y++)
                for (int x = margin; x < lw - margin; x++) {
                    const float v = D1.at(x, y);
                    if (!(v > cfg.hessian_threshold)) continue;
                    const FImg* N[3] = {&D0, &D1, &D2};
                    auto n9 = [&](int i, int dy, int dx) { return N[i]->at(x + dx, y + dy); };
                    bool mx = true;
                    for (int i = 0; i < 3 && mx; i++)
                        for (int dy = -1; dy <= 1 && mx; dy++)
                            for (int dx = -1; dx <= 1; dx++) {
                                if (i == 1 && dx == 0 && dy == 0) continue;
                                if (!(v > n9(i, dy, dx))) {
                                    mx = false;
                                    break;
                                }
                            }
                    if (!mx) continue;
                    const int sum_y = step * (y - (size / 2) / step);
                    const int sum_x = step * (x - (size / 2) / step);
                    // trace at the sample (the reference reads its trace plane)
                    float dtmp, tr;
                    det_trace(sum, (x - L.mx) * step, (y - L.my) * step, L, &dtmp, &tr);
                    KeyPoint kp{fadd(float(sum_x), fmul(float(size - 1), 0.5f)),
                                fadd(float(sum_y), fmul(float(size - 1), 0.5f)),
                                float(size),
                                -1.0f,
                                v,
                                o,
                                tr > 0 ? 1 : 0};
                    // interpolateKeypoint (SURF.metal:207-247)
                    const float B[3] = {-fdiv(fsub(n9(1, 0, 1), n9(1, 0, -1)), 2.0f),
                                        -fdiv(fsub(n9(1, 1, 0), n9(1, -1, 0)), 2.0f),
                                        -fdiv(fsub(n9(2, 0, 0), n9(0, 0, 0)), 2.0f)};
                    const float dxx = fadd(fsub(n9(1, 0, -1), fmul(2.0f, n9(1, 0, 0))), n9(1, 0, 1));
                    const float dxy =
                        fdiv(fadd(fsub(fsub(n9(1, 1, 1), n9(1, 1, -1)), n9(1, -1, 1)), n9(1, -1, -1)), 4.0f);
                    const float dxs =
                        fdiv(fadd(fsub(fsub(n9(2, 0, 1), n9(2, 0, -1)), n9(0, 0, 1)), n9(0, 0, -1)), 4.0f);
                    const float dyy = fadd(fsub(n9(1, -1, 0), fmul(2.0f, n9(1, 0, 0))), n9(1, 1, 0));
                    const float dys =
                        fdiv(fadd(fsub(fsub(n9(2, 1, 0), n9(2, -1, 0)), n9(0, 1, 0)), n9(0, -1, 0)), 4.0f);
                    const float dss = fadd(fsub(n9(0, 0, 0), fmul(2.0f, n9(1, 0, 0))), n9(2, 0, 0));
                    const float A0[3] = {dxx, dxy, dxs}, A1[3] = {dxy, dyy, dys}, A2[3] = {dxs, dys, dss};
                    // solve3x3 (SURF.metal:189-205)
                    float X[3] = {0, 0, 0};
                    const float det = det3(A0, A1, A2);
                    if (det != 0.0f) {
                        X[2] = fdiv(det3(A0, A1, B), det);
                        if (cfg.per_axis_interp) {
                            X[0] = fdiv(det3(B, A1, A2), det);
                            X[1] = fdiv(det3(A0, B, A2), det);
                        } else {
                            X[0] = X[1] = X[2];
                        }
                    }
                    const bool all_zero = X[0] == 0.0f && X[1] == 0.0f && X[2] == 0.0f;
                    if (!all_zero && std::fabs(X[0]) <= 1.0f && std::fabs(X[1]) <= 1.0f && std::fabs(X[2]) <= 1.0f) {
                        kp.x = fadd(kp.x, fmul(X[0], float(step)));
                        kp.y = fadd(kp.y, fmul(X[1], float(step)));
                        kp.size = std::rint(fadd(kp.size, fmul(X[2], float(size - s0))));
                        kps.push_back(kp);
                    }
                }
        }
    std::sort(kps.begin(), kps.end(), keypoint_greater);
    return kps;
}

// ------------------------------------------------------------ descriptors
// getGaussianKernel (SURF.cpp:394-425) for sigma > 0, as the reference
// evaluates it (float exp of a float argument; double scale, then float).
inline std::vector<float> gaussian_kernel(int n, float sigma) {
    const float sigmaX = sigma;
    const float scale2X = float(-0.5 / double(sigmaX * sigmaX));
    float sum = 0;
    std::vector<float> k(n);
    for (int i = 0; i < n; i++) {
        const float x = float(i - (n - 1) * 0.5);
        k[i] = std::exp(scale2X * x * x);
        sum += k[i];
    }
    sum = float(1. / sum);
    for (auto& v : k) v *= sum;
    return k;
}

struct DescriptorTables {  // SURFInvoker constructor (SURF.cpp:466-497)
    int n_ori = 0;
    float apt_x[169], apt_y[169], aptw[169];
    float dw[400];
};

inline DescriptorTables descriptor_tables() {
    DescriptorTables t;
    const auto g = gaussian_kernel(13, 2.5f);
    for (int i = -6; i <= 6; i++)
        for (int j = -6; j <= 6; j++)
            if (i * i + j * j <= 36) {
                t.apt_x[t.n_ori] = float(i);
                t.apt_y[t.n_ori] = float(j);
                t.aptw[t.n_ori++] = g[i + 6] * g[j + 6];
            }
    const auto gd = gaussian_kernel(20, 3.3f);
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) t.dw[i * 20 + j] = gd[i] * gd[j];
    return t;
}

// integralRectangle of SURF.cpp:79-82: the 0.5 is a double literal, so the
// expression is evaluated in double and rounded once.
inline float rect_cpu(float tr, float tl, float br, float bl) {
    return float((0.5 + double(fsub(tr, tl))) - double(fsub(br, bl)));
}

// calcHaarPattern (SURF.cpp:84-101) over boxes given as corner points
// p = {(x1,y1), (x1,y2), (x2,y1), (x2,y2)}
template <size_t N>
inline float haar_cpu(const FImg& sum, int px, int py, const std::array<HaarBox, N>& f) {
    float d = 0;
    for (size_t k = 0; k < N; k++) {
        const HaarBox& b = f[k];
        const float p0 = sum.at(px + b.x1, py + b.y1), p1 = sum.at(px + b.x1, py + b.y2);
        const float p2 = sum.at(px + b.x2, py + b.y1), p3 = sum.at(px + b.x2, py + b.y2);
        d = fadd(d, fmul(b.w, rect_cpu(p0, p1, p2, p3)));
    }
    return d;
}

// SURFInvoker::computeRange (SURF.cpp:499-677) for one keypoint: the
// dominant orientation (kp.angle, in radians as the reference stores it)
// and the 64-D descriptor, with the reference's quirks kept: the window
// rotation converts the radian angle as if it were degrees (:611), window
// pixels sampled inside the image are rounded to integers (:629), and
// resizeVV's third tap reads src[_j][_j + 1] (:441). A keypoint whose
// wavelet does not fit or whose orientation samples all fall outside gets
// size -1 and an all-zero descriptor.
inline void describe(const FImg& img, const FImg& sum, const DescriptorTables& T, KeyPoint& kp, float* desc) {
    for (int k = 0; k < 64; k++) desc[k] = 0.0f;
    const float size = kp.size;
    const float s = fdiv(fmul(size, 1.2f), 9.0f);
    const int grad_wav_size = 2 * int(std::lrint(fmul(2.0f, s)));
    if (sum.h < grad_wav_size || sum.w < grad_wav_size) {
        kp.size = -1;
        return;
    }
    static const int dx_s[2][5] = {{0, 0, 2, 4, -1}, {2, 0, 4, 4, 1}};
    static const int dy_s[2][5] = {{0, 0, 4, 2, 1}, {0, 2, 4, 4, -1}};
    const auto dx_t = resize_haar<2>(dx_s, 4, grad_wav_size);
    const auto dy_t = resize_haar<2>(dy_s, 4, grad_wav_size);
    float X[169], Y[169], ang[169];
    int nangle = 0;
    const float half_wav = fdiv(float(grad_wav_size - 1), 2.0f);
    for (int kk = 0; kk < T.n_ori; kk++) {
        const int x = int(std::lrint(fsub(fadd(kp.x, fmul(T.apt_x[kk], s)), half_wav)));
        const int y = int(std::lrint(fsub(fadd(kp.y, fmul(T.apt_y[kk], s)), half_wav)));
        if (y < 0 || y >= sum.h - grad_wav_size || x < 0 || x >= sum.w - grad_wav_size) continue;
        const float vx = haar_cpu<2>(sum, x, y, dx_t);
        const float vy = haar_cpu<2>(sum, x, y, dy_t);
        X[nangle] = fmul(vx, T.aptw[kk]);
        Y[nangle] = fmul(vy, T.aptw[kk]);
        nangle++;
    }
    if (nangle == 0) {
        kp.size = -1;
        return;
    }
    for (int i = 0; i < nangle; i++) {
        const float t = float(double(glsm::gls_atan2f(Y[i], X[i])) * (180 / M_PI));
        ang[i] = t < 0 ? fadd(t, 360.0f) : t;
    }
    float bestx = 0, besty = 0, best_mod = 0;
    for (int b = 0; b < 72; b++) {
        const float i = float(5 * b);  // the float loop counter is exact
        float sx = 0, sy = 0;
        for (int j = 0; j < nangle; j++) {
            const float d = std::fabs(fsub(float(std::lrint(ang[j])), i));
            if (d < 30.0f || d > 330.0f) {
                sx = fadd(sx, X[j]);
                sy = fadd(sy, Y[j]);
            }
        }
        const float m = fadd(fmul(sx, sx), fmul(sy, sy));
        if (m > best_mod) {
            best_mod = m;
            bestx = sx;
            besty = sy;
        }
    }
    float dir = glsm::gls_atan2f(-besty, bestx);
    kp.angle = dir;

    const int win = int(fmul(21.0f, s));
    dir = fmul(dir, float(M_PI / 180));
    const float sin_dir = -glsm::gls_sinf(dir);
    const float cos_dir = glsm::gls_cosf(dir);
    const float off = -fdiv(float(win - 1), 2.0f);
    float start_x = fadd(fadd(kp.x, fmul(off, cos_dir)), fmul(off, sin_dir));
    float start_y = fadd(fsub(kp.y, fmul(off, sin_dir)), fmul(off, cos_dir));
    const int ncols1 = img.w - 1, nrows1 = img.h - 1;
    std::vector<float> mwin(size_t(win) * win);
    for (int i = 0; i < win; i++, start_x = fadd(start_x, sin_dir), start_y = fadd(start_y, cos_dir)) {
        float px = start_x, py = start_y;
        for (int j = 0; j < win; j++, px = fadd(px, cos_dir), py = fsub(py, sin_dir)) {
            const int ix = int(std::floor(px)), iy = int(std::floor(py));
            float v;
            if (unsigned(ix) < unsigned(ncols1) && unsigned(iy) < unsigned(nrows1)) {
                const float a = fsub(px, float(ix)), b = fsub(py, float(iy));
                const float oa = fsub(1.0f, a), ob = fsub(1.0f, b);
                const float top = fadd(fmul(img.at(ix, iy), oa), fmul(img.at(ix + 1, iy), a));
                const float bot = fadd(fmul(img.at(ix, iy + 1), oa), fmul(img.at(ix + 1, iy + 1), a));
                v = std::round(fadd(fmul(top, ob), fmul(bot, b)));
            } else {
                const int x = std::clamp(int(std::round(px)), 0, ncols1);
                const int y = std::clamp(int(std::round(py)), 0, nrows1);
                v = img.at(x, y);
            }
            mwin[size_t(i) * win + j] = v;
        }
    }
    // resizeVV (SURF.cpp:427-446) to 21 x 21
    float P[21][21] = {};
    const float dsize = fdiv(float(win), 21.0f);
    for (int i = 0; i < 21; i++)
        for (int j = 0; j < 21; j++) {
            const float fi = fmul(float(i), dsize), fj = fmul(float(j), dsize);
            const int ii = int(fi), jj = int(fj);
            const float id = fsub(fi, float(ii)), jd = fsub(fj, float(jj));
            if (jj >= 0 && jj < win - 1 && ii >= 0 && ii < win - 1) {
                auto M = [&](int r, int c) { return mwin[size_t(r) * win + c]; };
                const float oi = fsub(1.0f, id), oj = fsub(1.0f, jd);
                float v = fmul(fmul(oi, oj), M(ii, jj));
                v = fadd(v, fmul(fmul(id, oj), M(ii + 1, jj)));
                v = fadd(v, fmul(fmul(jd, oi), M(jj, jj + 1)));
                v = fadd(v, fmul(fmul(id, jd), M(ii + 1, jj + 1)));
                P[i][j] = v;
            }
        }
    float DX[20][20], DY[20][20];
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) {
            const float dw = T.dw[i * 20 + j];
            DX[i][j] = fmul(fsub(fadd(fsub(P[i][j + 1], P[i][j]), P[i + 1][j + 1]), P[i + 1][j]), dw);
            DY[i][j] = fmul(fsub(fadd(fsub(P[i + 1][j], P[i][j]), P[i + 1][j + 1]), P[i][j + 1]), dw);
        }
    float sq = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            const int idx = 16 * i + 4 * j;
            for (int y = i * 5; y < i * 5 + 5; y++)
                for (int x = j * 5; x < j * 5 + 5; x++) {
                    const float tx = DX[y][x], ty = DY[y][x];
                    desc[idx + 0] = fadd(desc[idx + 0], tx);
                    desc[idx + 1] = fadd(desc[idx + 1], ty);
                    desc[idx + 2] = fadd(desc[idx + 2], std::fabs(tx));
                    desc[idx + 3] = fadd(desc[idx + 3], std::fabs(ty));
                }
            for (int k = 0; k < 4; k++) sq = fadd(sq, fmul(desc[idx + k], desc[idx + k]));
        }
    const float scale = float(1. / double(fadd(glsm::fsqrt(sq), FLT_EPSILON)));
    for (int k = 0; k < 64; k++) desc[k] = fmul(desc[k], scale);
}

// SURFInvoker::run (SURF.cpp:681-693): with more than 32 keypoints the
// reference cuts them into ceil(K / 8) ranges of ceil(K / 8) keypoints, so
// only the first min(K, ceil(K / 8)^2) are oriented and described; the
// others keep angle -1 and an all-zero descriptor (K = 33..56 loses some).
// With per_axis_interp (the corrected detector) every keypoint is.
inline int described_keypoints(int k, bool all) {
    if (all || k <= 32) return k;
    const int r = (k + 7) / 8;
    return std::min(k, r * r);
}

// detectAndCompute (SURF.cpp:1380-1450) with one section: integral,
// detection, the max_features cut, orientation and descriptors.
struct Features {
    std::vector<KeyPoint> kps;
    std::vector<float> desc;  // [n][64]
};

inline Features detect_and_compute(const FImg& img, const SurfConfig& cfg) {
    const FImg sum = integral(img);
    Features f;
    f.kps = detect(sum, img.w, img.h, cfg);
    if (cfg.max_features >= 0 && int(f.kps.size()) > cfg.max_features) f.kps.resize(cfg.max_features);
    f.desc.assign(f.kps.size() * 64, 0.0f);
    const DescriptorTables T = descriptor_tables();
    const int nd = described_keypoints(int(f.kps.size()), cfg.per_axis_interp);
    parallel_rows(nd, [&](int k) { describe(img, sum, T, f.kps[k], &f.desc[size_t(k) * 64]); });
    return f;
}

// ------------------------------------------------------------ matching
struct Match {
    int query, train;
    float distance;
};

// L2Norm over float4 lanes (SURF.metal:423-431)
inline float l2_lanes(const float* a, const float* b) {
    float s[4] = {0, 0, 0, 0};
    for (int g = 0; g < 16; g++)
        for (int l = 0; l < 4; l++) {
            const float d = fsub(a[4 * g + l], b[4 * g + l]);
            s[l] = fadd(s[l], fmul(d, d));
        }
    return glsm::fsqrt(fadd(fadd(fadd(s[0], s[1]), s[2]), s[3]));
}

// matchKeyPoints (SURF.metal:441-487) with 24 lanes per query, then
// refineMatch ordering (SURF.cpp:917-929, 971).
inline std::vector<Match> match(const std::vector<float>& d1, int n1, const std::vector<float>& d2, int n2) {
    std::vector<Match> m(n1);
    parallel_rows(n1, [&](int i) {
        float lane_d[24];
        int lane_j[24];
        for (int lid = 0; lid < 24; lid++) {
            float dmin = FLT_MAX;
            int jmin = 0;
            for (int j = 0; j + lid < n2; j += 24) {
                const float d = l2_lanes(&d1[size_t(i) * 64], &d2[size_t(j + lid) * 64]);
                if (d < dmin) {
                    dmin = d;
                    jmin = j + lid;
                }
            }
            lane_d[lid] = dmin;
            lane_j[lid] = jmin;
        }
        float dmin = lane_d[0];
        int jmin = lane_j[0];
        for (int l = 1; l < 24; l++)
            if (lane_d[l] < dmin) {
                dmin = lane_d[l];
                jmin = lane_j[l];
            }
        m[i] = {i, jmin, dmin};
    });
    std::sort(m.begin(), m.end(), [](const Match& a, const Match& b) {
        if (a.distance < b.distance) return true;
        if (a.distance > b.distance) return false;
        return a.query < b.query;
    });
    return m;
}

// ------------------------------------------------------------ homography
using Mat3f = std::array<float, 9>;
using Mat9d = std::array<double, 81>;

inline double hypot_d(double a, double b) { return glsm::dsqrt(glsm::dadd(glsm::dmul(a, a), glsm::dmul(b, b))); }

// Jacobi eigen-solver for a symmetric 9x9 matrix (LeastSquaresHomography.cpp
// :218-353): the largest-pivot cyclic Jacobi with row/column pivot indices,
// eigenvalues sorted descending; V holds eigenvectors as rows.
inline void jacobi9(const Mat9d& A, double W[9], Mat9d& V) {
    constexpr int N = 9;
    Mat9d a = A;
    const double eps = DBL_EPSILON;
    for (int i = 0; i < N * N; i++) V[i] = 0;
    for (int i = 0; i < N; i++) V[i * N + i] = 1;
    int indR[N] = {}, indC[N] = {};
    auto upd = [&](int k) {
        if (k < N - 1) {
            int m = k + 1;
            double mv = std::fabs(a[k * N + m]);
            for (int i = k + 2; i < N; i++) {
                const double val = std::fabs(a[k * N + i]);
                if (mv < val) mv = val, m = i;
            }
            indR[k] = m;
        }
        if (k > 0) {
            int m = 0;
            double mv = std::fabs(a[k]);
            for (int i = 1; i < k; i++) {
                const double val = std::fabs(a[i * N + k]);
                if (mv < val) mv = val, m = i;
            }
            indC[k] = m;
        }
    };
    for (int k = 0; k < N; k++) {
        W[k] = a[k * N + k];
        upd(k);
    }
    auto rot = [](double& v0, double& v1, double c, double s) {
        const double a0 = v0, b0 = v1;
        v0 = glsm::dsub(glsm::dmul(a0, c), glsm::dmul(b0, s));
        v1 = glsm::dadd(glsm::dmul(a0, s), glsm::dmul(b0, c));
    };
    for (int it = 0; it < N * N * 30; it++) {
        int k = 0;
        double mv = std::fabs(a[indR[0]]);
        for (int i = 1; i < N - 1; i++) {
            const double val = std::fabs(a[i * N + indR[i]]);
            if (mv < val) mv = val, k = i;
        }
        int l = indR[k];
        for (int i = 1; i < N; i++) {
            const double val = std::fabs(a[indC[i] * N + i]);
            if (mv < val) mv = val, k = indC[i], l = i;
        }
        const double p = a[k * N + l];
        if (std::fabs(p) <= eps) break;
        const double y = glsm::dmul(glsm::dsub(W[l], W[k]), 0.5);
        double t = glsm::dadd(std::fabs(y), hypot_d(p, y));
        double s = hypot_d(p, t);
        const double c = glsm::ddiv(t, s);
        s = glsm::ddiv(p, s);
        t = glsm::dmul(glsm::ddiv(p, t), p);
        if (y < 0) {
            s = -s;
            t = -t;
        }
        a[k * N + l] = 0;
        W[k] = glsm::dsub(W[k], t);
        W[l] = glsm::dadd(W[l], t);
        for (int i = 0; i < k; i++) rot(a[i * N + k], a[i * N + l], c, s);
        for (int i = k + 1; i < l; i++) rot(a[k * N + i], a[i * N + l], c, s);
        for (int i = l + 1; i < N; i++) rot(a[k * N + i], a[l * N + i], c, s);
        for (int i = 0; i < N; i++) rot(V[k * N + i], V[l * N + i], c, s);
        upd(k);
        upd(l);
    }
    for (int k = 0; k < N - 1; k++) {
        int m = k;
        for (int i = k + 1; i < N; i++)
            if (W[m] < W[i]) m = i;
        if (k != m) {
            std::swap(W[m], W[k]);
            for (int i = 0; i < N; i++) std::swap(V[m * N + i], V[k * N + i]);
        }
    }
}

// FindLeastSquaresHomography (LeastSquaresHomography.cpp:355-423): Hartley
// normalisation by centroid and mean absolute deviation, the 9x9 normal
// matrix accumulated upper-triangular in double, its least eigenvector,
// de-normalised and scaled so H[2][2] = 1. Returns false where the
// reference throws (a degenerate point spread).
inline bool ls_homography(const float* p1, const float* p2, int n, Mat3f& H) {
    using namespace glsm;
    double cM[2] = {0, 0}, cm[2] = {0, 0}, sM[2] = {0, 0}, sm[2] = {0, 0};
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 2; c++) {
            cm[c] = dadd(cm[c], double(p2[2 * i + c]));
            cM[c] = dadd(cM[c], double(p1[2 * i + c]));
        }
    for (int c = 0; c < 2; c++) {
        cm[c] = ddiv(cm[c], double(n));
        cM[c] = ddiv(cM[c], double(n));
    }
    for (int i = 0; i < n; i++)
        for (int c = 0; c < 2; c++) {
            sm[c] = dadd(sm[c], std::fabs(dsub(double(p2[2 * i + c]), cm[c])));
            sM[c] = dadd(sM[c], std::fabs(dsub(double(p1[2 * i + c]), cM[c])));
        }
    for (int c = 0; c < 2; c++) {
        sm[c] = ddiv(sm[c], double(n));
        sM[c] = ddiv(sM[c], double(n));
    }
    const double eps = DBL_EPSILON;
    if (std::fabs(sm[0]) < eps || std::fabs(sm[1]) < eps || std::fabs(sM[0]) < eps || std::fabs(sM[1]) < eps)
        return false;
    Mat9d L{};
    for (int i = 0; i < n; i++) {
        const double a0 = ddiv(dsub(double(p1[2 * i]), cM[0]), sM[0]);
        const double a1 = ddiv(dsub(double(p1[2 * i + 1]), cM[1]), sM[1]);
        const double b0 = ddiv(dsub(double(p2[2 * i]), cm[0]), sm[0]);
        const double b1 = ddiv(dsub(double(p2[2 * i + 1]), cm[1]), sm[1]);
        const double Lx[9] = {a0, a1, 1, 0, 0, 0, dmul(-b0, a0), dmul(-b0, a1), -b0};
        const double Ly[9] = {0, 0, 0, a0, a1, 1, dmul(-b1, a0), dmul(-b1, a1), -b1};
        for (int j = 0; j < 9; j++)
            for (int k = j; k < 9; k++) L[j * 9 + k] = dadd(L[j * 9 + k], dadd(dmul(Lx[j], Lx[k]), dmul(Ly[j], Ly[k])));
    }
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < i; j++) L[i * 9 + j] = L[j * 9 + i];  // completeSymm
    double W[9];
    Mat9d V;
    jacobi9(L, W, V);
    const double* h0 = &V[8 * 9];
    // invHnorm * H0 * Hnorm2, row-major products summed left to right
    const double inv[9] = {sm[0], 0, cm[0], 0, sm[1], cm[1], 0, 0, 1};
    const double nrm[9] = {ddiv(1, sM[0]), 0, ddiv(-cM[0], sM[0]), 0, ddiv(1, sM[1]), ddiv(-cM[1], sM[1]), 0, 0, 1};
    double T[9], R[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc = dadd(acc, dmul(inv[i * 3 + k], h0[k * 3 + j]));
            T[i * 3 + j] = acc;
        }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double acc = 0;
            for (int k = 0; k < 3; k++) acc = dadd(acc, dmul(T[i * 3 + k], nrm[k * 3 + j]));
            R[i * 3 + j] = acc;
        }
    const float d = float(R[8]);
    for (int i = 0; i < 9; i++) H[i] = fdiv(float(R[i]), d);
    return true;
}

// applyHomography + squared error (Homography.cpp:65-70): float.
inline float homography_error(const Mat3f& H, float x1, float y1, float x2, float y2) {
    const float w = fadd(fadd(fmul(H[6], x1), fmul(H[7], y1)), H[8]);
    const float u = fdiv(fadd(fadd(fmul(H[0], x1), fmul(H[1], y1)), H[2]), w);
    const float v = fdiv(fadd(fadd(fmul(H[3], x1), fmul(H[4], y1)), H[5]), w);
    const float dx = fsub(u, x2), dy = fsub(v, y2);
    return fadd(fmul(dx, dx), fmul(dy, dy));
}

// RTL::RANSAC::GenerateModel's sample sets (RTL/RANSAC.hpp:95-99): per
// iteration, draws into a std::set until it holds 4 indices; returned in
// the set's ascending order.
template <class Draw>
inline std::vector<std::array<int, 4>> ransac_samples(int iterations, Draw&& draw) {
    std::vector<std::array<int, 4>> out(iterations);
    for (int it = 0; it < iterations; it++) {
        std::set<int> s;
        while (s.size() < 4) s.insert(draw());
        int k = 0;
        for (int v : s) out[it][k++] = v;
    }
    return out;
}

// mask-and-reject uniform integer in [0, n-1] over a 32-bit engine
inline std::vector<std::array<int, 4>> ransac_samples_mask(int iterations, int n) {
    std::mt19937 g;
    const uint32_t range = uint32_t(n);
    int w = 0;
    while (w < 32 && (uint64_t(1) << w) < range) w++;
    const uint32_t mask = w >= 32 ? 0xffffffffu : ((1u << w) - 1u);
    return ransac_samples(iterations, [&]() {
        if (range <= 1) return 0;
        uint32_t u;
        do {
            u = uint32_t(g()) & mask;
        } while (u >= range);
        return int(u);
    });
}

inline std::vector<std::array<int, 4>> ransac_samples_std(int iterations, int n) {
    std::mt19937 g;
    std::uniform_int_distribution<int> u(0, n - 1);
    return ransac_samples(iterations, [&]() { return u(g); });
}

// FindHomography (Homography.cpp:72-116) over RTL::RANSAC::FindBest /
// FindInliers (RTL/RANSAC.hpp:47-77): every iteration fits the 4-point
// model (identity when degenerate), counts errors above the threshold
// (NaN errors do not count), keeps the first strictly better model; the
// inliers (|error| < threshold) are refitted by least squares when there
// are at least 4 of them.
struct HomographyResult {
    Mat3f H;
    std::vector<int> inliers;
    float loss;
};

inline HomographyResult find_homography(const float* p1, const float* p2, int n, float threshold,
                                        const std::vector<std::array<int, 4>>& samples) {
    HomographyResult r;
    r.H = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float best = HUGE_VALF;
    for (const auto& smp : samples) {
        float a[8], b[8];
        for (int k = 0; k < 4; k++) {
            a[2 * k] = p1[2 * smp[k]];
            a[2 * k + 1] = p1[2 * smp[k] + 1];
            b[2 * k] = p2[2 * smp[k]];
            b[2 * k + 1] = p2[2 * smp[k] + 1];
        }
        Mat3f H;
        if (!ls_homography(a, b, 4, H)) H = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        float loss = 0;
        for (int i = 0; i < n; i++) {
            const float e = homography_error(H, p1[2 * i], p1[2 * i + 1], p2[2 * i], p2[2 * i + 1]);
            loss = fadd(loss, std::fabs(e) > threshold ? 1.0f : 0.0f);
        }
        if (loss < best) {
            best = loss;
            r.H = H;
        }
    }
    r.loss = best;
    for (int i = 0; i < n; i++) {
        const float e = homography_error(r.H, p1[2 * i], p1[2 * i + 1], p2[2 * i], p2[2 * i + 1]);
        if (std::fabs(e) < threshold) r.inliers.push_back(i);
    }
    if (r.inliers.size() >= 4) {
        std::vector<float> a, b;
        for (int i : r.inliers) {
            a.push_back(p1[2 * i]);
            a.push_back(p1[2 * i + 1]);
            b.push_back(p2[2 * i]);
            b.push_back(p2[2 * i + 1]);
        }
        Mat3f H;
        if (ls_homography(a.data(), b.data(), int(r.inliers.size()), H)) r.H = H;
    }
    return r;
}

// ScaleHomography (ImageRegistration/Homography.hpp:29-37): S H S^-1 with
// S = diag(2, 2, 1) whatever the scale argument.
inline Mat3f scale_homography(const Mat3f& H) {
    return {H[0], H[1], fmul(H[2], 2.0f), H[3], H[4], fmul(H[5], 2.0f), fmul(H[6], 0.5f), fmul(H[7], 0.5f), H[8]};
}

// ------------------------------------------------------------ warps
// registerAndFuse (SURF.metal:489-516): out = ((count-1) fused + warped) / count
inline void register_and_fuse(const float* fused, const float* input, int w, int h, const Mat3f& H, int count,
                              float* out) {
    parallel_rows(h, [&](int y) {
        for (int x = 0; x < w; x++) {
            const float fx = float(x), fy = float(y);
            const float u = fadd(fadd(fmul(H[0], fx), fmul(H[1], fy)), H[2]);
            const float v = fadd(fadd(fmul(H[3], fx), fmul(H[4], fy)), H[5]);
            const float ww = fadd(fadd(fmul(H[6], fx), fmul(H[7], fy)), H[8]);
            // clamp to [-1, size]: the same samples under clamp-to-edge, and
            // a defined edge sample for non-finite coordinates
            const float xx = fminf(fmaxf(fdiv(u, ww), -1.0f), float(w));
            const float yy = fminf(fmaxf(fdiv(v, ww), -1.0f), float(h));
            float s[4];
            const float x0f = std::floor(xx), y0f = std::floor(yy);
            const float ax = fsub(xx, x0f), ay = fsub(yy, y0f);
            const int x0 = int(x0f), y0 = int(y0f);
            auto rd = [&](int X, int Y, int c) {
                X = std::clamp(X, 0, w - 1);
                Y = std::clamp(Y, 0, h - 1);
                return input[(size_t(Y) * w + X) * 4 + c];
            };
            for (int c = 0; c < 4; c++) {
                const float t = fadd(rd(x0, y0, c), fmul(ax, fsub(rd(x0 + 1, y0, c), rd(x0, y0, c))));
                const float b = fadd(rd(x0, y0 + 1, c), fmul(ax, fsub(rd(x0 + 1, y0 + 1, c), rd(x0, y0 + 1, c))));
                s[c] = fadd(t, fmul(ay, fsub(b, t)));
            }
            const float* f = &fused[(size_t(y) * w + x) * 4];
            float* o = &out[(size_t(y) * w + x) * 4];
            const float cm1 = float(count - 1), cn = float(count);
            for (int c = 0; c < 4; c++) o[c] = fdiv(fadd(fmul(cm1, f[c]), s[c]), cn);
        }
    });
}

}  // namespace reg
}  // namespace orc
