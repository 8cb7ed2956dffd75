// oracle_reg_capi.cpp — TEST INFRASTRUCTURE ONLY. extern "C" entry points of
// the registration oracle (gls_oracle_reg.hpp) for the pytest suite, called
// through ctypes. Keypoints use the library's gls_keypoint layout
// (include/glscam.h), which is the reference's KeyPoint (feature2d.hpp:25-47).
#include "../include/glscam.h"
#include "gls_oracle_reg.hpp"

using namespace orc::reg;

static_assert(sizeof(gls_keypoint) == sizeof(KeyPoint), "keypoint layouts differ");

extern "C" {

// 0: atan2f(a, b), 1: sinf(a), 2: cosf(a) with the library's own functions
void orc_reg_math(int fn, const float* a, const float* b, float* out, int n) {
    for (int i = 0; i < n; i++)
        out[i] = fn == 0 ? glsm::gls_atan2f(a[i], b[i]) : fn == 1 ? glsm::gls_sinf(a[i]) : glsm::gls_cosf(a[i]);
}

int orc_reg_raw_channel(const uint16_t* raw, int w, int h, size_t stride_px, int pattern, int c, float black,
                        float white, float exposure, float* out) {
    if (pattern < 0 || pattern > 3 || c < 0 || c > 3) return -1;
    const FImg img = raw_channel(raw, w, h, stride_px, pattern, c, black, white, exposure);
    std::copy(img.d.begin(), img.d.end(), out);
    return 0;
}

int orc_reg_integral(const float* in, int w, int h, float* sum) {
    FImg img(w, h);
    std::copy(in, in + size_t(w) * h, img.d.begin());
    const FImg s = integral(img);
    std::copy(s.d.begin(), s.d.end(), sum);
    return 0;
}

// detectAndCompute; returns the number of keypoints written (<= capacity)
// and the total before the max_features cut in *n_found
int orc_reg_detect(const float* in, int w, int h, int n_octaves, int n_layers, float threshold, int max_features,
                   gls_keypoint* kps, float* desc, int capacity, int* n_found, int per_axis_interp) {
    FImg img(w, h);
    std::copy(in, in + size_t(w) * h, img.d.begin());
    SurfConfig cfg;
    cfg.n_octaves = n_octaves;
    cfg.n_octave_layers = n_layers;
    cfg.hessian_threshold = threshold;
    cfg.max_features = -1;
    cfg.per_axis_interp = per_axis_interp != 0;
    const FImg sum = integral(img);
    std::vector<KeyPoint> all = detect(sum, w, h, cfg);
    if (n_found) *n_found = int(all.size());
    if (max_features >= 0 && int(all.size()) > max_features) all.resize(max_features);
    const DescriptorTables T = descriptor_tables();
    std::vector<float> d(all.size() * 64);
    const int nd = described_keypoints(int(all.size()), cfg.per_axis_interp);
    orc::parallel_rows(nd, [&](int k) { describe(img, sum, T, all[k], &d[size_t(k) * 64]); });
    const int n = std::min(int(all.size()), capacity);
    std::memcpy(kps, all.data(), size_t(n) * sizeof(KeyPoint));
    if (desc) std::copy(d.begin(), d.begin() + size_t(n) * 64, desc);
    return n;
}

// orientation + descriptor of given keypoints over an image (kps updated)
int orc_reg_describe(const float* in, int w, int h, gls_keypoint* kps, int n, float* desc) {
    FImg img(w, h);
    std::copy(in, in + size_t(w) * h, img.d.begin());
    const FImg sum = integral(img);
    const DescriptorTables T = descriptor_tables();
    auto* k = reinterpret_cast<KeyPoint*>(kps);
    orc::parallel_rows(n, [&](int i) { describe(img, sum, T, k[i], &desc[size_t(i) * 64]); });
    return 0;
}

int orc_reg_match(const float* d1, int n1, const float* d2, int n2, gls_match* out) {
    std::vector<float> a(d1, d1 + size_t(n1) * 64), b(d2, d2 + size_t(n2) * 64);
    const auto m = match(a, n1, b, n2);
    for (int i = 0; i < n1; i++) out[i] = {m[i].query, m[i].train, m[i].distance};
    return n1;
}

int orc_reg_ls_homography(const float* p1, const float* p2, int n, float* H) {
    Mat3f m;
    if (!ls_homography(p1, p2, n, m)) return -1;
    std::copy(m.begin(), m.end(), H);
    return 0;
}

// sampler 0: mask-and-reject (the product's), 1: this toolchain's
// std::uniform_int_distribution
int orc_reg_samples(int iterations, int n, int sampler, int* out) {
    const auto s = sampler == 0 ? ransac_samples_mask(iterations, n) : ransac_samples_std(iterations, n);
    for (int i = 0; i < iterations; i++)
        for (int k = 0; k < 4; k++) out[4 * i + k] = s[i][k];
    return 0;
}

int orc_reg_find_homography(const float* p1, const float* p2, int n, float threshold, int iterations, int sampler,
                            float* H, int* inliers, int* n_inliers, float* loss) {
    if (n <= 0) return -1;
    const auto s = sampler == 0 ? ransac_samples_mask(iterations, n) : ransac_samples_std(iterations, n);
    const auto r = find_homography(p1, p2, n, threshold, s);
    std::copy(r.H.begin(), r.H.end(), H);
    if (inliers)
        for (size_t i = 0; i < r.inliers.size(); i++) inliers[i] = r.inliers[i];
    if (n_inliers) *n_inliers = int(r.inliers.size());
    if (loss) *loss = r.loss;
    return 0;
}

void orc_reg_scale_homography(const float* H, float* out) {
    Mat3f m;
    std::copy(H, H + 9, m.begin());
    const Mat3f r = scale_homography(m);
    std::copy(r.begin(), r.end(), out);
}

int orc_reg_fuse(const float* fused, const float* input, int w, int h, const float* H, int count, float* out) {
    Mat3f m;
    std::copy(H, H + 9, m.begin());
    register_and_fuse(fused, input, w, h, m, count, out);
    return 0;
}

}  // extern "C"
