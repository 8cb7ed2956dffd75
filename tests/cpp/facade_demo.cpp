// facade_demo.cpp — exercises include/glscam.hpp the way a caller of the
// reference's C++ API would: calibration -> RawConverter::demosaic with
// noise reduction -> SURF on a shifted pair -> FindHomography; then a DNG
// file -> parameters from its metadata -> demosaic with post-processing,
// and findBursts. Prints
// "facade ok" and exits 0 when every result is sane.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "glscam.hpp"

int main() {
    const int W = 256, H = 192;
    std::vector<uint16_t> raw(size_t(W) * H);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const double v = 0.3 + 0.2 * std::sin(x * 0.07) * std::cos(y * 0.05) + ((x / 32 + y / 32) % 2) * 0.2;
            raw[size_t(y) * W + x] = uint16_t(512 + v * (4095 - 512));
        }
    gls::iPhone14WideCalibration<4> cal;
    gls::DemosaicParameters p = cal.getDemosaicParameters(400);
    p.bayer_pattern = GLS_RGGB;
    p.black_level = 512;
    p.white_level = 4095;
    p.exposure_multiplier = 1;
    for (int c = 0; c < 4; c++) p.scale_mul[c] = 65535.0f / (4095 - 512);
    for (int i = 0; i < 9; i++) p.rgb_cam[i] = (i % 4 == 0) ? 1.0f : 0.0f;
    const float xyz[9] = {0.4124f, 0.3576f, 0.1805f, 0.2126f, 0.7152f, 0.0722f, 0.0193f, 0.1192f, 0.9505f};
    for (int i = 0; i < 9; i++) p.xyz_rgb[i] = xyz[i];
    for (int c = 0; c < 4; c++) {
        p.raw_nlf.a[c] = 1e-6f;
        p.raw_nlf.b[c] = 2e-4f;
    }

    gls::RawConverter conv(0);
    std::vector<float> rgb(size_t(W) * H * 4);
    gls::ImageView out{rgb.data(), W, H, 4, GLS_F32, size_t(W) * 16};
    conv.demosaic(raw.data(), W, H, size_t(W) * 2, &p, &out, /*noiseReduction=*/true, /*fp16=*/false,
                  /*host_io=*/true);
    double mean = 0;
    for (size_t i = 0; i < rgb.size(); i += 4) {
        if (!std::isfinite(rgb[i])) {
            std::printf("non-finite output\n");
            return 1;
        }
        mean += rgb[i];
    }
    mean /= double(W) * H;

    // SURF on an image and its 3 px / 5 px shifted copy
    const int SW = 320, SH = 240;
    std::vector<float> a(size_t(SW) * SH), b(size_t(SW) * SH);
    for (int y = 0; y < SH; y++)
        for (int x = 0; x < SW; x++) {
            auto f = [](double u, double v) {
                double s = 0.6;
                for (int k = 0; k < 40; k++) {
                    const double cx = 17 + (k * 73) % 290, cy = 13 + (k * 37) % 215, r = 3 + k % 7;
                    if ((u - cx) * (u - cx) + (v - cy) * (v - cy) < r * r) s = 0.1 + 0.02 * (k % 5);
                }
                return s;
            };
            a[size_t(y) * SW + x] = float(f(x, y));
            b[size_t(y) * SW + x] = float(f(x - 5, y - 3));
        }
    gls::SURF surf = gls::SURF::makeInstance(SW, SH, 1500);
    std::vector<gls::KeyPoint> k1, k2;
    std::vector<float> d1, d2;
    const int s1 = surf.detectAndCompute(a.data(), SW, SH, size_t(SW) * 4, &k1, &d1, /*host_input=*/true);
    const int s2 = surf.detectAndCompute(b.data(), SW, SH, size_t(SW) * 4, &k2, &d2, /*host_input=*/true);
    const auto matches = surf.findMatches(s1, k1, s2, k2);
    // the first frame's features as another GPU would receive them
    const int s1b = surf.loadFeatures(k1, d1);
    const auto m_direct = surf.matchKeyPoints(s1, s2), m_loaded = surf.matchKeyPoints(s1b, s2);
    bool loaded_ok = m_direct.size() == m_loaded.size();
    for (size_t i = 0; loaded_ok && i < m_direct.size(); i++)
        loaded_ok = m_direct[i].train_idx == m_loaded[i].train_idx && m_direct[i].distance == m_loaded[i].distance;
    std::vector<int> inliers;
    const auto Hm = gls::FindHomography(surf, matches, 1.0f, 2000, &inliers);
    const bool shift_ok = std::fabs(Hm[2] - 5) < 0.5 && std::fabs(Hm[5] - 3) < 0.5;
    std::printf("mean luma %.4f, keypoints %zu/%zu, matches %zu, inliers %zu, H shift (%.3f, %.3f)\n", mean,
                k1.size(), k2.size(), matches.size(), inliers.size(), Hm[2], Hm[5]);
    bool range_thrown = false;
    try {
        cal.getDemosaicParameters(0);  // not a valid ISO
    } catch (const std::range_error&) {
        range_thrown = true;
    }
    if (!(mean > 0.05 && mean < 1.5) || k1.empty() || !shift_ok || !range_thrown || !loaded_ok) {
        std::printf("facade check failed\n");
        return 1;
    }

    // the file path: a DNG written and read back, parameters from its
    // metadata, demosaic with display post-processing into host memory
    gls_dng_info info{};
    info.width = W;
    info.height = H;
    const uint8_t rggb[4] = {0, 1, 1, 2};
    for (int c = 0; c < 4; c++) info.cfa_pattern[c] = rggb[c];
    info.black_level = 512;
    info.white_level = 4095;
    info.iso = 400;
    info.has_color_matrix2 = 1;
    const float cm[9] = {0.66f, -0.13f, -0.07f, -0.39f, 1.21f, 0.17f, -0.06f, 0.17f, 0.55f};
    for (int k = 0; k < 9; k++) info.color_matrix2[k] = cm[k];
    const std::string path = "facade_demo_frame.dng";
    gls::check(gls_dng_write(path.c_str(), &info, raw.data(), size_t(W), 7, 64));
    gls_dng_info back{};
    const std::vector<uint16_t> raw2 = gls::read_dng_file(path, &back);
    std::remove(path.c_str());
    gls::iPhone14WideCalibration<5> cal5;
    gls::DemosaicParameters pd = cal5.getDemosaicParameters(back, xyz);
    std::vector<float> srgb(size_t(W) * H * 4);
    gls::ImageView sout{srgb.data(), W, H, 4, GLS_F32, size_t(W) * 16};
    conv.demosaic(raw2.data(), W, H, size_t(W) * 2, &pd, &sout, /*noiseReduction=*/true, /*fp16=*/true,
                  /*host_io=*/true, nullptr, /*postProcess=*/true);
    bool srgb_ok = raw2 == raw && back.iso == 400;
    for (size_t i = 0; i < srgb.size(); i++) srgb_ok = srgb_ok && srgb[i] >= 0.f && srgb[i] <= 1.f;
    const auto bursts = gls::findBursts({"d/A_1_x.dng", "d/A_2_x.dng", "d/B.dng", "d/C_1_y.dng"});
    const bool bursts_ok = bursts.size() == 2 && bursts[0].size() == 2 && bursts[1].size() == 1;
    std::printf("dng round trip %s, sRGB in range %s, bursts %zu\n", raw2 == raw ? "exact" : "differs",
                srgb_ok ? "yes" : "no", bursts.size());
    if (!srgb_ok || !bursts_ok) {
        std::printf("facade check failed\n");
        return 1;
    }
    std::printf("facade ok\n");
    return 0;
}
