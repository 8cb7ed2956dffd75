// oracle_capi.cpp — TEST INFRASTRUCTURE ONLY. extern "C" entry points of the
// CPU oracle (gls_oracle.hpp) for the pytest suite and the CPU-baseline leg
// of bench.py, called through ctypes. Parameters arrive in the library's own
// gls_demosaic_params layout (include/glscam.h) so that both sides read one
// struct. Parity of the oracle: see the header of gls_oracle.hpp.
#include <chrono>
#include <cstdio>

#include "../include/glscam.h"
#include "gls_oracle.hpp"
#include "gls_oracle_nlf.hpp"
#include "gls_oracle_post.hpp"

using namespace orc;

static Params to_params(const gls_demosaic_params* g) {
    Params p;
    p.bayer = g->bayer_pattern;
    p.black = g->black_level;
    p.white = g->white_level;
    p.lsc = g->lens_shading_correction;
    for (int c = 0; c < 4; c++) p.scale_mul[c] = g->scale_mul[c];
    for (int i = 0; i < 9; i++) {
        p.rgb_cam[i] = g->rgb_cam[i];
        p.xyz_rgb[i] = g->xyz_rgb[i];
    }
    p.high_noise = g->high_noise_image != 0;
    p.raw_strength = g->raw_denoise_strength;
    for (int c = 0; c < 4; c++) {
        p.raw_nlf.a[c] = g->raw_nlf.a[c];
        p.raw_nlf.b[c] = g->raw_nlf.b[c];
    }
    for (int l = 0; l < 5; l++) {
        for (int c = 0; c < 3; c++) {
            p.pyr_nlf[l].a[c] = g->pyramid_nlf[l].a[c];
            p.pyr_nlf[l].b[c] = g->pyramid_nlf[l].b[c];
        }
        p.dn[l].luma = g->denoise[l].luma;
        p.dn[l].chroma = g->denoise[l].chroma;
        p.dn[l].chromaBoost = g->denoise[l].chroma_boost;
        p.dn[l].gradientBoost = g->denoise[l].gradient_boost;
        p.dn[l].gradientThreshold = g->denoise[l].gradient_threshold;
        p.dn[l].sharpening = g->denoise[l].sharpening;
    }
    p.levels = g->levels;
    return p;
}

template <class T, int C>
static void copy_out(const Img<T, C>& img, float* dst) {
    if (!dst) return;
    for (size_t i = 0; i < img.d.size(); i++) dst[i] = float(img.d[i]);
}

template <class T, int C>
static Img<T, C> copy_in(const float* src, int w, int h) {
    Img<T, C> img(w, h);
    for (size_t i = 0; i < img.d.size(); i++) img.d[i] = T(src[i]);
    return img;
}

template <class T>
static void run_pipeline(const uint16_t* raw, int w, int h, size_t stride, const gls_demosaic_params* gp,
                         int denoise, float* out, float* scaled, float* grad, float* demosaiced,
                         float* despeckled, double* bases) {
    const Params p = to_params(gp);
    Stages st;
    st.keep = scaled || grad || demosaiced || despeckled;
    PyramidOut info;
    auto res = raw_pipeline<T>(raw, stride, w, h, p, denoise != 0, &st, &info);
    copy_out(res, out);
    if (st.keep) {
        copy_out(st.scaled, scaled);
        copy_out(st.gradient, grad);
        copy_out(st.demosaiced, demosaiced);
        if (denoise) copy_out(st.despeckled, despeckled);
    }
    if (bases && denoise) {
        for (size_t l = 0; l < info.bases.size(); l++)
            for (int r = 0; r < 25; r++)
                for (int c = 0; c < 8; c++) bases[(l * 25 + r) * 8 + c] = info.bases[l][r][c];
    }
}

extern "C" {

void orc_set_threads(int n) { num_threads() = n > 0 ? n : 1; }
int orc_get_threads(void) { return num_threads(); }

// RawConverter::demosaic on the CPU. f64 selects the double "truth" run.
// Optional outputs may be NULL: scaled (w*h), grad (w*h*2), demosaiced and
// despeckled (w*h*4), bases (levels*25*8 doubles).
int orc_raw_pipeline(const uint16_t* raw, int w, int h, size_t stride_elems, const gls_demosaic_params* p,
                     int denoise, int f64, float* out_rgba, float* scaled, float* grad, float* demosaiced,
                     float* despeckled, double* bases) {
    if (!raw || !p || w < 2 || h < 2 || p->levels < 1 || p->levels > 5) return 1;
    if (f64)
        run_pipeline<double>(raw, w, h, stride_elems, p, denoise, out_rgba, scaled, grad, demosaiced, despeckled, bases);
    else
        run_pipeline<float>(raw, w, h, stride_elems, p, denoise, out_rgba, scaled, grad, demosaiced, despeckled, bases);
    return 0;
}

// PyramidProcessor::denoise on the CPU, from a YCbCr RGBA image and a 2-ch
// gradient. den_levels (optional) receives the denoised level images packed
// one after the other (4 ch each, level sizes w>>i x h>>i).
int orc_pyramid_denoise(const float* ycc, const float* grad, int w, int h, const gls_demosaic_params* gp, int f64,
                        float* out, float* den_levels, double* bases) {
    const Params p = to_params(gp);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        auto img = copy_in<T, 4>(ycc, w, h);
        auto g = copy_in<T, 2>(grad, w, h);
        std::vector<Plane4<T>> levels;
        PyramidOut info;
        auto res = pyramid_denoise<T>(img, g, p, &levels, &info);
        copy_out(res, out);
        if (den_levels) {
            size_t off = 0;
            for (auto& l : levels) {
                copy_out(l, den_levels + off);
                off += l.d.size();
            }
        }
        if (bases)
            for (size_t l = 0; l < info.bases.size(); l++)
                for (int r = 0; r < 25; r++)
                    for (int c = 0; c < 8; c++) bases[(l * 25 + r) * 8 + c] = info.bases[l][r][c];
    };
    if (f64) run(double());
    else run(float());
    return 0;
}

// MSE of the FP64 pyramid denoise + output transform against a target,
// with the per-level PCA bases given (held fixed): the function whose
// central differences check the adjoint. y2c: YCbCr -> camera RGB, 3x3
// row-major; target: h x w x tch floats (RGB first).
int orc_pyramid_loss(const float* ycc, const float* grad, int w, int h, const gls_demosaic_params* gp,
                     const double* bases, const double* y2c, const float* target, int tch, double* loss) {
    const Params p = to_params(gp);
    std::vector<std::array<std::array<double, 8>, 25>> fb(p.levels);
    for (int l = 0; l < p.levels; l++)
        for (int r = 0; r < 25; r++)
            for (int c = 0; c < 8; c++) fb[l][r][c] = bases[(l * 25 + r) * 8 + c];
    auto img = copy_in<double, 4>(ycc, w, h);
    auto g = copy_in<double, 2>(grad, w, h);
    const auto den = pyramid_denoise<double>(img, g, p, nullptr, nullptr, &fb);
    double acc = 0;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const double* d = den.px(x, y);
            const float* t = target + (size_t(y) * w + x) * tch;
            for (int r = 0; r < 3; r++) {
                const double o = y2c[r * 3 + 0] * d[0] + y2c[r * 3 + 1] * d[1] + y2c[r * 3 + 2] * d[2];
                acc += (o - t[r]) * (o - t[r]);
            }
        }
    *loss = acc / (3.0 * double(w) * h);
    return 0;
}

// ---- single stages from given inputs (for the stage-by-stage pin against
// the reference's own kernels, oracle/ref_harness.cpp)

int orc_scale(const uint16_t* raw, int w, int h, const gls_demosaic_params* gp, int f64, float* scaled) {
    const Params p = to_params(gp);
    if (f64) copy_out(scale_raw<double>(raw, w, w, h, p), scaled);
    else copy_out(scale_raw<float>(raw, w, w, h, p), scaled);
    return 0;
}

int orc_sobel_blur(const float* scaled, int w, int h, const gls_demosaic_params* gp, int f64, float* grad) {
    const Params p = to_params(gp);
    static const Taps t1 = gaussian_bilinear_taps(1.5f), t2 = gaussian_bilinear_taps(4.5f);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        auto s = copy_in<T, 1>(scaled, w, h);
        copy_out(gradient_blur(s, sobel(s), t1, t2, raw_variance(p.raw_nlf)[1]), grad);
    };
    if (f64) run(double());
    else run(float());
    return 0;
}

int orc_raw_denoise(const float* scaled, const float* grad, int w, int h, const gls_demosaic_params* gp, int f64,
                    float* scaled_out) {
    const Params p = to_params(gp);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        auto s = copy_in<T, 1>(scaled, w, h);
        auto g = copy_in<T, 2>(grad, w, h);
        auto rgba = bayer_to_rgba(s, p.bayer);
        auto ds = despeckle_raw_rgba(rgba, g, p.raw_nlf.b);
        auto cd = cross_denoise_raw_rgba(ds, p.raw_nlf.b, p.raw_strength);
        rgba_to_bayer(cd, p.bayer, s);
        copy_out(s, scaled_out);
    };
    if (f64) run(double());
    else run(float());
    return 0;
}

int orc_demosaic_rgb(const float* scaled, const float* grad, int w, int h, const gls_demosaic_params* gp, int f64,
                     float* rgb) {
    const Params p = to_params(gp);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        auto s = copy_in<T, 1>(scaled, w, h);
        auto g = copy_in<T, 2>(grad, w, h);
        auto out = demosaic(s, g, p.bayer, raw_variance(p.raw_nlf));
        blend_highlights(out, T(1));
        copy_out(out, rgb);
    };
    if (f64) run(double());
    else run(float());
    return 0;
}

int orc_despeckle(const float* ycc, int w, int h, const gls_demosaic_params* gp, int f64, float* out) {
    const Params p = to_params(gp);
    auto run = [&](auto tag) {
        using T = decltype(tag);
        copy_out(despeckle_luma_median_chroma(copy_in<T, 4>(ycc, w, h), p.pyr_nlf[0].a, p.pyr_nlf[0].b), out);
    };
    if (f64) run(double());
    else run(float());
    return 0;
}

int orc_gaussian_taps(float radius, float* taps, int max_taps, int* n) {
    Taps t = gaussian_bilinear_taps(radius);
    *n = int(t.t.size());
    if (int(t.t.size()) > max_taps) return 1;
    for (size_t i = 0; i < t.t.size(); i++)
        for (int k = 0; k < 3; k++) taps[i * 3 + k] = t.t[i][k];
    return 0;
}

void orc_cam_ycbcr(const float* rgb_cam, const float* xyz_rgb, float* fwd, float* inv) {
    Mat3 m = cam_ycbcr(rgb_cam, xyz_rgb);
    Mat3 mi = inverse3(m);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            fwd[i * 3 + j] = m.m[i][j];
            inv[i * 3 + j] = mi.m[i][j];
        }
}

// Bayer quad pack then unpack (bayerToRawRGBA o rawRGBAToBayer), identity.
int orc_bayer_roundtrip(const float* raw, int w, int h, int pattern, float* rgba, float* back) {
    auto img = copy_in<float, 1>(raw, w, h);
    auto q = bayer_to_rgba(img, pattern);
    copy_out(q, rgba);
    Plane<float> b(w, h);
    rgba_to_bayer(q, pattern, b);
    copy_out(b, back);
    return 0;
}

// Pyramid downsample of a C-channel float image (C = 2 or 4).
int orc_downsample(const float* in, int w, int h, int ch, int ow, int oh, int f64, float* out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        if (ch == 4) copy_out(downsample<T, 4>(copy_in<T, 4>(in, w, h), ow, oh, 4), out);
        else copy_out(downsample<T, 2>(copy_in<T, 2>(in, w, h), ow, oh, 2), out);
    };
    if (ch != 2 && ch != 4) return 1;
    if (f64) run(double());
    else run(float());
    return 0;
}

// PCA basis (25 x 8, row-major) of the luma of a 4-channel float image.
int orc_pca_basis(const float* img4, int w, int h, double* basis) {
    auto img = copy_in<double, 4>(img4, w, h);
    auto b = pca_basis(img);
    for (int r = 0; r < 25; r++)
        for (int c = 0; c < 8; c++) basis[r * 8 + c] = b[r][c];
    return 0;
}

// Symmetric eigen-decomposition (values descending, vectors as columns).
int orc_jacobi(int n, const double* a, double* evals, double* evecs) {
    std::vector<double> m(a, a + size_t(n) * n), v;
    jacobi_eigen(n, m, v);
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return m[x * n + x] > m[y * n + y]; });
    for (int c = 0; c < n; c++) {
        evals[c] = m[idx[c] * n + idx[c]];
        for (int r = 0; r < n; r++) evecs[r * n + c] = v[r * n + idx[c]];
    }
    return 0;
}


// The display post-processing (gls_oracle_post.hpp) of one frame from its
// denoised levels (5 levels packed, 4 ch, sizes w >> l x h >> l; NULL
// without noise reduction), level-0 gradient (2 ch) and linear camera RGB
// (4 ch); seed = the raw frame's first pixel. stats (optional, 6 floats):
// black, white, shadows, highlights, mean, median.
int orc_postprocess(const float* den_levels, const float* grad, const float* rgb, int w, int h,
                    const gls_demosaic_params* gp, unsigned seed, int f64, float* out, float* stats) {
    if (!grad || !rgb || !gp || !out || w < 16 || h < 16) return 1;
    post::PostParams pp;
    const gls_rgb_conversion_params& rc = gp->rgb_conversion;
    pp.contrast = rc.contrast;
    pp.saturation = rc.saturation;
    pp.slope = rc.tone_curve_slope;
    pp.bias = rc.exposure_bias + std::log2(gp->exposure_multiplier);
    pp.blacks = rc.blacks;
    pp.ltm = rc.local_tone_mapping != 0;
    pp.eps = gp->ltm.eps;
    for (int k = 0; k < 3; k++) pp.detail[k] = gp->ltm.detail[k];
    pp.nlf[0] = gp->pyramid_nlf[0].a[0];
    pp.nlf[1] = gp->pyramid_nlf[0].b[0];
    pp.luma_var[0] = 2.0f * ((gp->raw_nlf.a[1] + gp->raw_nlf.a[3]) / 2);
    pp.luma_var[1] = 2.0f * ((gp->raw_nlf.b[1] + gp->raw_nlf.b[3]) / 2);
    for (int i = 0; i < 9; i++) pp.rgb_cam[i] = gp->rgb_cam[i];
    auto run = [&](auto tag) {
        using T = decltype(tag);
        std::vector<Plane4<T>> den;
        if (den_levels) {
            size_t off = 0;
            for (int l = 0; l < 5; l++) {
                den.push_back(copy_in<T, 4>(den_levels + off, w >> l, h >> l));
                off += size_t(w >> l) * (h >> l) * 4;
            }
        }
        const auto g = copy_in<T, 2>(grad, w, h);
        const auto c = copy_in<T, 4>(rgb, w, h);
        post::Stats st;
        const auto o = post::postprocess<T>(den, g, c, pp, seed, &st);
        copy_out(o, out);
        if (stats) {
            const float v[6] = {st.black, st.white, st.shadows, st.highlights, st.mean, st.median};
            std::copy(v, v + 6, stats);
        }
    };
    if (f64) run(double());
    else run(float());
    return 0;
}
// ---- noise-model measurement (calibrateFromImage), FP32 statistics ----

// basicRawNoiseStatistics: mean, var are (w/2) x (h/2) x 4
int orc_raw_noise_stats(const float* scaled, int w, int h, int pattern, float* mean, float* var) {
    if (!scaled || !mean || !var || w < 2 || h < 2 || pattern < 0 || pattern > 3) return 1;
    const auto s = copy_in<float, 1>(scaled, w, h);
    Plane4<float> m, v;
    nlf::raw_stats(s, pattern, m, v);
    copy_out(m, mean);
    copy_out(v, var);
    return 0;
}

// basicNoiseStatistics: stats is w x h x 4 (mean Y, var Y, var Cb, var Cr)
int orc_ycc_noise_stats(const float* img, int w, int h, float* stats) {
    if (!img || !stats || w < 1 || h < 1) return 1;
    copy_out(nlf::ycc_stats(copy_in<float, 4>(img, w, h)), stats);
    return 0;
}

int orc_measure_raw_nlf(const float* mean, const float* var, int raw_w, int raw_h, float exposure_multiplier,
                        float* a, float* b) {
    if (!mean || !var || !a || !b || raw_w < 2 || raw_h < 2) return 1;
    const RawNLF r = nlf::measure_raw(copy_in<float, 4>(mean, raw_w / 2, raw_h / 2),
                                      copy_in<float, 4>(var, raw_w / 2, raw_h / 2), raw_w, raw_h, exposure_multiplier);
    std::copy(r.a, r.a + 4, a);
    std::copy(r.b, r.b + 4, b);
    return 0;
}

int orc_measure_ycc_nlf(const float* stats, int w, int h, float exposure_multiplier, float* a, float* b) {
    if (!stats || !a || !b || w < 1 || h < 1) return 1;
    const YCbCrNLF r = nlf::measure_ycc(copy_in<float, 4>(stats, w, h), exposure_multiplier);
    std::copy(r.a, r.a + 3, a);
    std::copy(r.b, r.b + 3, b);
    return 0;
}

// RawConverter::demosaic with calibrateFromImage and noise reduction: out
// RGBA (w = 0); raw_nlf (8 floats: a[4], b[4]) and pyr_nlf (levels x 6:
// a[3], b[3]) receive the measured models.
int orc_raw_pipeline_calibrated(const uint16_t* raw, int w, int h, size_t stride_elems, const gls_demosaic_params* gp,
                                int f64, float* out_rgba, float* raw_nlf, float* pyr_nlf) {
    if (!raw || !gp || !out_rgba || w < 2 || h < 2 || gp->levels < 1 || gp->levels > 5) return 1;
    const Params p = to_params(gp);
    RawNLF mr{};
    YCbCrNLF mp[5]{};
    auto run = [&](auto tag) {
        using T = decltype(tag);
        copy_out(nlf::raw_pipeline_calibrated<T>(raw, stride_elems, w, h, p, gp->exposure_multiplier, &mr, mp),
                 out_rgba);
    };
    if (f64) run(double());
    else run(float());
    if (raw_nlf) {
        std::copy(mr.a, mr.a + 4, raw_nlf);
        std::copy(mr.b, mr.b + 4, raw_nlf + 4);
    }
    if (pyr_nlf)
        for (int l = 0; l < p.levels; l++) {
            std::copy(mp[l].a, mp[l].a + 3, pyr_nlf + 6 * l);
            std::copy(mp[l].b, mp[l].b + 3, pyr_nlf + 6 * l + 3);
        }
    return 0;
}

}  // extern "C"
