// ref_reg_harness.cpp — TEST INFRASTRUCTURE ONLY. Runs the reference's own
// registration code on the CPU as the pin of the registration oracle
// (gls_oracle_reg.hpp). Built by `make -C oracle ref` into
// oracle/_ref/libglsref_reg.so from unmodified line ranges of the reference
// sources, which the recipe extracts into oracle/_ref/ (not committed):
//   SURF.metal       :17-40, 64-559   every kernel, under metal_shim/, in
//                                     ref_reg_metal.cpp
//   SURF.cpp         :29, 37-128      Haar patterns, CPU integral
//                    :200-320         gpuSurfHF, DetAndTraceHaarPattern
//                    :394-706         Gaussian kernel, resizeVV, SURFInvoker
//                                     (orientation and descriptor)
//                    :917-929         refineMatch
//                    :1215-1227       KeypointGreater
//                    :1298-1383       mergeKeypoints
//   LeastSquaresHomography.cpp :189-423   Jacobi + FindLeastSquaresHomography
//   Homography.cpp   :23-24, 37-116   FindHomography over RTL::RANSAC
// and the headers SURF.hpp, Homography.hpp, LeastSquaresHomography.hpp,
// feature2d.hpp and RTL/ included where they lie. GlassImage, which those
// sources include, is not in the reference tree; gls_shim/ stands in for it.
//
// Left out: SURF.cpp:129-199 and 321-393, the CPU detector's solve3x3,
// interpolateKeypoint and findMaximaInLayer. The stock build detects on the
// GPU (USE_GPU_HESSIAN_DETECTOR, SURF.cpp:31), and that solve3x3 returns a
// gls::Vector from a bool function, which only the absent GlassImage can
// convert.
//
// Restated here, not taken from the reference:
//   * the Metal host side of SURFGPU (SURF.cpp:776-975, 1082-1290,
//     1385-1471): buffer and texture set-up and the dispatch grids, written
//     out below with the line each step follows.
// Threadgroups of the integral and matching kernels run as groups of host
// threads sharing their `threadgroup` arrays, with a real barrier.
//
// Semantics the Metal and C sources leave to the platform:
//   * SURF.metal:200 `(float3)(a, b, c)` is C++ (Metal is a C++14 dialect):
//     a cast of the comma expression, i.e. float3(c). solve3x3 therefore
//     returns the scale offset in all three lanes (ref_reg_metal.cpp).
//   * atan2 in SURF.cpp (unqualified, inside namespace gls) is the float
//     atan2f of the platform's C library; hypot in the Jacobi solver is the
//     C library's. ref_reg_set_own_math(1) binds both to this library's own
//     functions instead (gls_atan2f, sqrt(a^2 + b^2) in double), the ones
//     the CUDA kernels and the oracle evaluate, so that the rest of the
//     arithmetic can be compared bit for bit.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include "ref_reg_metal.h"

#include "ThreadPool.hpp"
#include "feature2d.hpp"
#include "gls_geometry.hpp"
#include "gls_logging.h"
#include "SURF.hpp"
#include "Homography.hpp"
#include "LeastSquaresHomography.hpp"
#include "RTL/RTL.hpp"

#include "../glasscamerapublic_b200/csrc/gls_fmath.h"

// ------------------------------------------------- SURF.cpp / homography code
namespace gls {
static int g_own_math = 0;

inline float atan2(float y, float x) { return g_own_math ? glsm::gls_atan2f(y, x) : ::atan2f(y, x); }
inline double hypot(double a, double b) { return g_own_math ? std::sqrt(a * a + b * b) : ::hypot(a, b); }

#include "surf_cpu.inc"
#include "lsh.inc"
#include "homography.inc"
}  // namespace gls

namespace {

using metal::tex_fmt;
using metal::tex_store;

struct Plane {
    std::vector<float> px;
    tex_store st;
    Plane(int w, int h, int channels = 1) : px(size_t(w) * h * channels, 0.0f) {
        st.data = px.data();
        st.width = w;
        st.height = h;
        st.channels = channels;
        st.fmt = tex_fmt::f32;
    }
};

// A dispatch of `grid` threads in threadgroups of `group` (the last group
// may be smaller, as Metal's non-uniform dispatch makes it): one host thread
// per lane, groups one after another, each group's barrier installed for its
// threads. f(lane, group index, grid position).
template <class F>
void run_groups(int grid, int group, F&& f) {
    if (grid <= 0) return;
    const int ngroups = (grid + group - 1) / group;
    const int last_n = grid - (ngroups - 1) * group;
    metal::group_barrier full(group), last(last_n), outer(group);
    std::vector<std::thread> th;
    for (int l = 0; l < group; l++)
        th.emplace_back([&, l] {
            for (int g = 0; g < ngroups; g++) {
                const int n = g == ngroups - 1 ? last_n : group;
                if (l < n) {
                    metal::tg_barrier = n == group ? &full : &last;
                    f(l, g, g * group + l);
                    metal::tg_barrier = nullptr;
                }
                outer.arrive_and_wait();
            }
        });
    for (auto& t : th) t.join();
}

// A 2-D dispatch of a kernel without threadgroup memory, rows spread over
// the host's cores. f(x, y).
int g_threads = 0;
template <class F>
void run_rows(int w, int h, F&& f) {
    if (w <= 0 || h <= 0) return;
    const int nt = std::max(1, std::min(h, g_threads > 0 ? g_threads : int(std::thread::hardware_concurrency())));
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            for (int y = t; y < h; y += nt)
                for (int x = 0; x < w; x++) f(x, y);
        });
    for (auto& t : th) t.join();
}

struct RefSurf {
    int width, height, max_features, n_octaves = 4, n_octave_layers = 2;
    float threshold = 0.02f;
    static constexpr int kTile = 8;  // integralImageKernel::tileSize (SURF.cpp:779)

    // integralImageKernel (SURF.cpp:776-825): the four summed-area textures
    // of sumImageStack (SURF.cpp:708-717) for sampling steps 1, 2, 4, 8.
    // The textures and the column-sum buffer start out holding `fill`: the
    // kernels' non-uniform last threadgroups (gls_mtl.hpp:229-237 dispatches
    // with dispatchThreads) leave some entries unwritten when the width or
    // the height is not a multiple of 8, and Metal gives them no value.
    std::vector<std::unique_ptr<Plane>> integral(const gls::image<float>& img, float fill = 0.0f) const {
        const int w = img.width, h = img.height;
        Plane src(w, h);
        for (int y = 0; y < h; y++) std::memcpy(&src.px[size_t(y) * w], img[y], sizeof(float) * w);
        std::vector<std::unique_ptr<Plane>> sum;
        for (int step = 1; step <= 8; step *= 2) {
            sum.push_back(std::make_unique<Plane>(1 + w / step, 1 + h / step));
            std::fill(sum.back()->px.begin(), sum.back()->px.end(), fill);
        }
        // tmpSize = (rows rounded up to the tile, columns rounded up): a
        // transposed column-sum buffer of width tmp_w
        const int tmp_w = ((h + kTile - 1) / kTile) * kTile;
        const int tmp_h = ((w + kTile - 1) / kTile) * kTile;
        std::vector<float> tmp(size_t(tmp_w) * tmp_h, fill);
        run_groups(w, kTile, [&](int lid, int gid, int x) {
            refwrap::integral_sum_cols(&src.st, tmp.data(), tmp_w, unsigned(lid), unsigned(gid), unsigned(x));
        });
        run_groups(h, kTile, [&](int lid, int gid, int x) {
            refwrap::integral_sum_rows(tmp.data(), tmp_w, &sum[0]->st, &sum[1]->st, &sum[2]->st, &sum[3]->st,
                                       unsigned(lid), unsigned(gid), unsigned(h), unsigned(x));
        });
        return sum;
    }

    // SURFGPU::fastHessianDetector (SURF.cpp:1229-1286) with Build
    // (:1136-1165) and Find (:1173-1211) on the Metal kernels
    std::vector<KeyPoint> fast_hessian(const std::vector<std::unique_ptr<Plane>>& sum) const {
        const int layers = n_octave_layers + 2;
        const int total = layers * n_octaves;
        std::vector<int> sizes(total), steps(total), middle;
        for (int o = 0, idx = 0, step = 1; o < n_octaves; o++, step *= 2)
            for (int l = 0; l < layers; l++, idx++) {
                sizes[idx] = (9 + 6 * l) << o;  // SURF_HAAR_SIZE0 + SURF_HAAR_SIZE_INC * layer
                steps[idx] = step;
                if (0 < l && l <= n_octave_layers) middle.push_back(idx);
            }
        // det / trace textures per layer (SURFGPU constructor, SURF.cpp:1119-1133)
        std::vector<std::unique_ptr<Plane>> dets, traces;
        for (int i = 0; i < total; i++) {
            dets.push_back(std::make_unique<Plane>(width / steps[i], height / steps[i]));
            traces.push_back(std::make_unique<Plane>(width / steps[i], height / steps[i]));
        }
        for (int i = 0; i < total; i++) {  // Build: calcDetAndTraceKernel (SURF.cpp:827-863)
            const gls::DetAndTraceHaarPattern hp(sum[0]->st.width, sum[0]->st.height, sizes[i], steps[i]);
            const gls::gpuSurfHF hf(hp.Dx, hp.Dy, hp.Dxy);
            static_assert(sizeof(hf) == 256, "gpuSurfHF layout");
            run_rows(hp.margin_crop.width, hp.margin_crop.height, [&](int x, int y) {
                refwrap::calc_det_and_trace(&sum[0]->st, &dets[i]->st, &traces[i]->st, steps[i], hp.Dx[0].w,
                                            hp.Dxy[0].w, hp.margin_crop.x, hp.margin_crop.y, &hf, unsigned(x),
                                            unsigned(y));
            });
        }
        auto maxima = std::make_unique<refwrap::Maxima>();
        maxima->count = 0;
        for (size_t m = 0; m < middle.size(); m++) {  // Find: findMaximaInLayerKernel (SURF.cpp:876-915)
            const int layer = middle[m];
            const int octave = int(m) / n_octave_layers;
            const int step = steps[layer];
            const int lh = height / step, lw = width / step;
            const int margin = (sizes[layer + 1] / 2) / step + 1;
            // appended through the kernel's atomic counter in any order, then
            // sorted by KeypointGreater, a total order on distinct maxima
            run_rows(lw - 2 * margin, lh - 2 * margin, [&](int x, int y) {
                refwrap::find_maxima_in_layer(&dets[layer - 1]->st, &dets[layer]->st, &dets[layer + 1]->st,
                                              &traces[layer]->st, sizes[layer - 1], sizes[layer], sizes[layer + 1],
                                              maxima.get(), margin, octave, threshold, step, unsigned(x),
                                              unsigned(y));
            });
        }
        std::vector<KeyPoint> kps;
        const int n = std::min(maxima->count, refwrap::kMaximaCapacity);
        for (int i = 0; i < n; i++) {
            const auto& k = maxima->kp[i];
            kps.emplace_back(k.x, k.y, k.size, k.angle, k.response, k.octave, k.class_id);
        }
        std::sort(kps.begin(), kps.end(), gls::KeypointGreater());
        return kps;
    }

    // SURFGPU::detectAndCompute (SURF.cpp:1385-1471), one section
    void detect_and_compute(const gls::image<float>& img, std::vector<KeyPoint>* keypoints,
                            gls::image<float>::unique_ptr* descriptors, int* found) const {
        const gls::rectangle tile(0, 0, img.width, img.height);
        const auto tile_image = gls::image<float>(img, tile);
        const auto sum = integral(tile_image);
        auto tile_kps = std::make_unique<std::vector<KeyPoint>>(fast_hessian(sum));
        *found = int(tile_kps->size());
        if (tile_kps->size() > size_t(max_features))
            tile_kps->erase(tile_kps->begin() + max_features, tile_kps->end());
        const int n = int(tile_kps->size());
        auto tile_desc = std::make_unique<gls::image<float>>(64, n);
        gls::image<float> sum_cpu(sum[0]->st.width, sum[0]->st.height);
        for (int y = 0; y < sum_cpu.height; y++)
            std::memcpy(sum_cpu[y], &sum[0]->px[size_t(y) * sum_cpu.width], sizeof(float) * sum_cpu.width);
        gls::descriptor(tile_image, sum_cpu, tile_kps.get(), tile_desc.get());
        for (auto& kp : *tile_kps) kp.pt += Point2f(tile.x, tile.y);
        std::vector<std::unique_ptr<std::vector<KeyPoint>>> all_kps;
        std::vector<gls::image<float>::unique_ptr> all_desc;
        all_kps.push_back(std::move(tile_kps));
        all_desc.push_back(std::move(tile_desc));
        gls::mergeKeypoints(all_kps, keypoints, all_desc, descriptors);
    }
};

struct OutKeypoint {  // gls_keypoint
    float x, y, size, angle, response;
    int32_t octave, class_id;
};
struct OutMatch {  // gls_match
    int32_t query_idx, train_idx;
    float distance;
};

gls::image<float> wrap(const float* img, int w, int h) {
    gls::image<float> im(w, h);
    for (int y = 0; y < h; y++) std::memcpy(im[y], img + size_t(y) * w, sizeof(float) * w);
    return im;
}

}  // namespace

extern "C" {

void ref_reg_set_own_math(int on) { gls::g_own_math = on; }

// host threads for the per-pixel kernels (0 = all cores)
void ref_reg_set_threads(int n) { g_threads = n; }

// summed-area table, (h + 1) x (w + 1), of the integral kernels; entries
// the kernels never write are NaN
void ref_reg_integral(const float* img, int w, int h, float* out) {
    RefSurf s{w, h, -1};
    const auto sum = s.integral(wrap(img, w, h), std::numeric_limits<float>::quiet_NaN());
    std::memcpy(out, sum[0]->px.data(), sizeof(float) * size_t(w + 1) * (h + 1));
}

// SURF::detectAndCompute; returns the keypoint count (at most capacity
// written); *found receives the count before the max_features cut
int ref_reg_detect(const float* img, int w, int h, int n_octaves, int n_layers, float threshold, int max_features,
                   void* kps_out, float* desc_out, int capacity, int* found) {
    RefSurf s{w, h, max_features, n_octaves, n_layers, threshold};
    std::vector<KeyPoint> kps;
    gls::image<float>::unique_ptr desc;
    s.detect_and_compute(wrap(img, w, h), &kps, &desc, found);
    auto* o = static_cast<OutKeypoint*>(kps_out);
    const int n = std::min(int(kps.size()), capacity);
    for (int i = 0; i < n; i++) {
        o[i] = {kps[i].pt.x, kps[i].pt.y, kps[i].size, kps[i].angle, kps[i].response, kps[i].octave,
                kps[i].class_id};
        if (desc_out) std::memcpy(desc_out + size_t(i) * 64, (*desc)[i], 64 * sizeof(float));
    }
    return n;
}

// matchKeyPointsKernel (SURF.cpp:931-974): Metal matchKeyPoints over a
// (n1, 24) grid in (1, 24) threadgroups, then sorted by refineMatch
void ref_reg_match(const float* d1, int n1, const float* d2, int n2, void* out) {
    std::vector<float> a(64 * size_t(std::max(n1, 1))), b(64 * size_t(std::max(n2, 1)));
    std::memcpy(a.data(), d1, sizeof(float) * 64 * size_t(n1));
    std::memcpy(b.data(), d2, sizeof(float) * 64 * size_t(n2));
    std::vector<refwrap::Match> m(std::max(n1, 1));
    constexpr int kBlock = 24;  // match_block_size, SURF.cpp:937
    run_groups(n1 * kBlock, kBlock, [&](int lid, int gid, int) {
        refwrap::match_key_points(a.data(), b.data(), unsigned(n2), m.data(), unsigned(lid), unsigned(gid));
    });
    std::vector<gls::DMatch> r;
    for (int i = 0; i < n1; i++) r.emplace_back(int(m[i].query_idx), int(m[i].train_idx), m[i].distance);
    std::sort(r.begin(), r.end(), gls::refineMatch());
    auto* o = static_cast<OutMatch*>(out);
    for (int i = 0; i < n1; i++) o[i] = {r[i].queryIdx, r[i].trainIdx, r[i].distance};
}

// gls::FindHomography (Homography.cpp:72-116); returns the inlier count
// (at most capacity written)
int ref_reg_find_homography(const float* p1, const float* p2, int n, float threshold, int iterations, float* H,
                            int* inliers, int capacity) {
    std::vector<std::pair<Point2f, Point2f>> pts(n);
    for (int i = 0; i < n; i++)
        pts[i] = {Point2f(p1[2 * i], p1[2 * i + 1]), Point2f(p2[2 * i], p2[2 * i + 1])};
    std::vector<int> inl;
    const auto M = gls::FindHomography(pts, threshold, iterations, &inl);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H[i * 3 + j] = M[i][j];
    const int k = std::min(int(inl.size()), capacity);
    for (int i = 0; i < k; i++) inliers[i] = inl[i];
    return int(inl.size());
}

// gls::FindLeastSquaresHomography (LeastSquaresHomography.cpp:355-423);
// returns 0, or 1 where the reference throws std::range_error
int ref_reg_ls_homography(const float* p1, const float* p2, int n, float* H) {
    std::vector<Point2f> a(n), b(n);
    for (int i = 0; i < n; i++) {
        a[i] = Point2f(p1[2 * i], p1[2 * i + 1]);
        b[i] = Point2f(p2[2 * i], p2[2 * i + 1]);
    }
    try {
        const auto M = gls::FindLeastSquaresHomography(a, b);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) H[i * 3 + j] = M[i][j];
        return 0;
    } catch (const std::range_error&) {
        return 1;
    }
}

// gls::ScaleHomography (Homography.hpp:29-37)
void ref_reg_scale_homography(const float* H, float scale, float* out) {
    gls::Matrix<3, 3> M;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) M[i][j] = H[i * 3 + j];
    const auto S = gls::ScaleHomography(M, scale);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) out[i * 3 + j] = S[i][j];
}

// registerAndFuse (SURF.metal:493-516) over RGBA float planes
void ref_reg_fuse(const float* fused, const float* input, int w, int h, const float* H, int count, float* out) {
    Plane f(w, h, 4), in(w, h, 4), o(w, h, 4);
    std::memcpy(f.px.data(), fused, sizeof(float) * 4 * size_t(w) * h);
    std::memcpy(in.px.data(), input, sizeof(float) * 4 * size_t(w) * h);
    run_rows(w, h, [&](int x, int y) {
        refwrap::register_and_fuse(&f.st, &in.st, &o.st, H, count, unsigned(x), unsigned(y));
    });
    std::memcpy(out, o.px.data(), sizeof(float) * 4 * size_t(w) * h);
}

}  // extern "C"
