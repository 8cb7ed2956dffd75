// ref_harness.cpp — TEST INFRASTRUCTURE ONLY. Runs the reference's own Metal
// kernels (MetalPipeline/demosaic.metal, compiled as C++ against
// oracle/metal_shim/metal_stdlib) on the CPU, stage by stage, to pin the
// oracle. The recipe (oracle/Makefile, target ref) extracts two unmodified
// line ranges of demosaic.metal:
//   * lines 1-720    (helpers, raw scaling, Sobel, gradient blur, the three
//                     demosaic passes, highlights, colour transform), and
//   * lines 754-1291 (collectPatches, pcaProjection, blockMatchingDenoise,
//                     pyramid down/up-sampling and reconstruct, the
//                     high-noise quad kernels, despeckle and median);
//   * lines 1292-1723 (the display post-processing kernels);
// and this file supplies, between them, the `_half8` helper type and its
// `length` overloads of lines 721-752: eight halves bit-reinterpreted from
// and to uint4, element-wise subtraction, and a length over the first n
// lanes that squares in half and accumulates in float. (GCC rejects the
// reference's own declaration: class-type members in an anonymous struct,
// which Metal allows because its vectors are builtin types.)
//
// The host sequence around the kernels restates raw_converter.cpp:148-248,
// pyramid_processor.cpp:96-172 and, for post-processing,
// raw_converter.cpp:70-115 with demosaic_kernels.hpp:485-671; the grain
// tables come from the reference's own Noise2D (ref_noise.cpp). Two host pieces are the oracle's: the
// Gaussian tap folding (demosaic_utils.cpp:934-1006) and the PCA basis
// (Eigen in the reference; the oracle's FP64 Jacobi here, on the dense
// patch grid the reference's collectPatches kernel wrote), rounded to half
// as the reference stores pcaSpace.
#include "demosaic_a.inc"

struct _half8 {
    half4 hi, lo;
    _half8(half val) : hi(val), lo(val) {}
    _half8(int val) : hi(val), lo(val) {}
    explicit _half8(uint4 u) : hi((half4)u.xy), lo((half4)u.zw) {}
    _half8(half4 a, half4 b) : hi(a), lo(b) {}
    _half8 operator-(_half8 o) { return _half8(hi - o.hi, lo - o.lo); }
    operator uint4() const { return uint4(uint2(hi), uint2(lo)); }
    half at(int i) const { return i < 4 ? hi.d[i] : lo.d[i - 4]; }
};
static_assert(sizeof(_half8) == 16, "_half8 must be eight contiguous halves");

half length(_half8 x) {
    return sqrt(dot(x.hi, x.hi) + dot(x.lo, x.lo));
}

half length(_half8 x, int components) {
    float sum = 0;
    for (int i = 0; i < components; i++) {
        const half p = x.at(i) * x.at(i);
        sum += p;
    }
    return sqrt(sum);
}

#include "demosaic_b.inc"

// Lines 1292-1723 (the guided filter and box filter of local tone mapping,
// histogramImage / histogramStatistics, localToneMappingMaskImage, the
// Perlin grain and convertTosRGB) size arrays with `constant` scalars
// (histogramSize, noiseGradSize), so `constant` reads as `const` there.
#undef constant
#define constant const
#include "demosaic_c.inc"
#undef constant
#define constant

// ------------------------------------------------------------------ harness
#undef kernel
#undef device
#undef thread
#undef threadgroup
#undef constant

#include <thread>
#include <vector>

#include "../include/glscam.h"
#include "gls_oracle.hpp"

namespace ref {

template <class F>
void run_grid(int gw, int gh, F f) {
    orc::parallel_rows(gh, [&](int y) {
        for (int x = 0; x < gw; x++) f(metal::uint2(uint(x), uint(y)));
    });
}

struct Tex {
    std::vector<float> f;
    std::vector<uint16_t> u16;
    std::vector<uint32_t> u32;
    metal::tex_store st;
    Tex(int w, int h, int c, metal::tex_fmt fmt = metal::tex_fmt::f32) {
        st.width = w;
        st.height = h;
        st.channels = c;
        st.fmt = fmt;
        const size_t n = size_t(w) * h * c;
        if (fmt == metal::tex_fmt::f32) {
            f.assign(n, 0.f);
            st.data = f.data();
        } else if (fmt == metal::tex_fmt::unorm16) {
            u16.assign(n, 0);
            st.data = u16.data();
        } else {
            u32.assign(n, 0);
            st.data = u32.data();
        }
    }
    template <class T, metal::access A = metal::access::sample>
    metal::texture2d<T, A> t() {
        return metal::texture2d<T, A>(&st);
    }
};

static metal::float2 f2(float a, float b) { return metal::float2(a, b); }

}  // namespace ref

using namespace ref;
using metal::access;
using metal::half;

extern "C" {

// scaleRawData, raw_converter.cpp:179-183 (grid W/2 x H/2)
int ref_scale(const uint16_t* raw, int w, int h, const gls_demosaic_params* p, float* scaled) {
    Tex in(w, h, 1, metal::tex_fmt::unorm16), out(w, h, 1);
    std::copy(raw, raw + size_t(w) * h, in.u16.begin());
    int pattern = p->bayer_pattern;
    metal::half4 sm(half(p->scale_mul[0]), half(p->scale_mul[1]), half(p->scale_mul[2]), half(p->scale_mul[3]));
    half black = half(p->black_level / 65535.f);
    half lsc = half(p->lens_shading_correction);
    auto ti = in.t<half>();
    auto to = out.t<half, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { scaleRawData(ti, to, pattern, sm, black, lsc, i); });
    std::copy(out.f.begin(), out.f.end(), scaled);
    return 0;
}

// rawImageSobel + sampledConvolutionSobel, raw_converter.cpp:185-193
int ref_sobel_blur(const float* scaled, int w, int h, const gls_demosaic_params* p, float* grad) {
    Tex s(w, h, 1), sob(w, h, 4), g(w, h, 2);
    std::copy(scaled, scaled + size_t(w) * h, s.f.begin());
    auto ts_h = s.t<half>();
    auto tsob_w = sob.t<half, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { rawImageSobel(ts_h, tsob_w, i); });
    const orc::Taps t1 = orc::gaussian_bilinear_taps(1.5f), t2 = orc::gaussian_bilinear_taps(4.5f);
    std::vector<float> w1, w2;
    for (auto& t : t1.t) w1.insert(w1.end(), t.begin(), t.end());
    for (auto& t : t2.t) w2.insert(w2.end(), t.begin(), t.end());
    int n1 = int(t1.t.size()), n2 = int(t2.t.size());
    metal::float2 var = f2((p->raw_nlf.a[1] + p->raw_nlf.a[3]) / 2, (p->raw_nlf.b[1] + p->raw_nlf.b[3]) / 2);
    auto ts = s.t<float>();
    auto tsob = sob.t<float>();
    auto tg = g.t<float, access::write>();
    run_grid(w, h, [&](metal::uint2 i) {
        sampledConvolutionSobel(ts, tsob, n1, w1.data(), n2, w2.data(), var, tg, i);
    });
    std::copy(g.f.begin(), g.f.end(), grad);
    return 0;
}

// high-noise raw branch, raw_converter.cpp:195-202
int ref_raw_denoise(const float* scaled, const float* grad, int w, int h, const gls_demosaic_params* p,
                    float* scaled_out) {
    Tex s(w, h, 1), g(w, h, 2), q(w / 2, h / 2, 4), dq(w / 2, h / 2, 4);
    std::copy(scaled, scaled + size_t(w) * h, s.f.begin());
    std::copy(grad, grad + size_t(w) * h * 2, g.f.begin());
    int pattern = p->bayer_pattern;
    auto ts = s.t<float>();
    auto tq_w = q.t<float, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { bayerToRawRGBA(ts, tq_w, pattern, i); });
    metal::float4 var4(p->raw_nlf.b[0], p->raw_nlf.b[1], p->raw_nlf.b[2], p->raw_nlf.b[3]);
    auto tq_h = q.t<half>();
    auto tg_h = g.t<half>();
    auto tdq_w = dq.t<half, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { despeckleRawRGBAImage(tq_h, tg_h, var4, tdq_w, i); });
    metal::half4 varh(half(p->raw_nlf.b[0]), half(p->raw_nlf.b[1]), half(p->raw_nlf.b[2]), half(p->raw_nlf.b[3]));
    half strength = half(p->raw_denoise_strength);
    auto tdq_h = dq.t<half>();
    auto tq_hw = q.t<half, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { crossDenoiseRawRGBAImage(tdq_h, varh, strength, tq_hw, i); });
    auto tq = q.t<float>();
    auto ts_w = s.t<float, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { rawRGBAToBayer(tq, ts_w, pattern, i); });
    std::copy(s.f.begin(), s.f.end(), scaled_out);
    return 0;
}

// demosaicImageKernel (demosaic_kernels.hpp:154-180) + blendHighlightsImage (clip 1)
int ref_demosaic_rgb(const float* scaled, const float* grad, int w, int h, const gls_demosaic_params* p, float* rgb) {
    Tex s(w, h, 1), g(w, h, 2), green(w, h, 1), tmp(w, h, 4), out(w, h, 4);
    std::copy(scaled, scaled + size_t(w) * h, s.f.begin());
    std::copy(grad, grad + size_t(w) * h * 2, g.f.begin());
    int pattern = p->bayer_pattern;
    metal::float2 rv = f2(p->raw_nlf.a[0], p->raw_nlf.b[0]);
    metal::float2 gv = f2((p->raw_nlf.a[1] + p->raw_nlf.a[3]) / 2, (p->raw_nlf.b[1] + p->raw_nlf.b[3]) / 2);
    metal::float2 bv = f2(p->raw_nlf.a[2], p->raw_nlf.b[2]);
    auto ts = s.t<float>();
    auto tg = g.t<float>();
    auto tgreen_w = green.t<float, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { interpolateGreen(ts, tg, tgreen_w, pattern, gv, i); });
    auto tgreen = green.t<float>();
    auto ttmp_w = tmp.t<float, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { interpolateRedBlue(ts, tgreen, tg, ttmp_w, pattern, rv, bv, i); });
    auto ttmp = tmp.t<float>();
    auto tout_w = out.t<float, access::write>();
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { interpolateRedBlueAtGreen(ttmp, tg, tout_w, pattern, rv, bv, i); });
    float clip = 1.0f;
    auto tout = out.t<float>();
    run_grid(w, h, [&](metal::uint2 i) { blendHighlightsImage(tout, clip, tout_w, i); });
    std::copy(out.f.begin(), out.f.end(), rgb);
    return 0;
}

// transformImage with a row-major 3x3 matrix
int ref_transform(const float* in, int w, int h, const float* m9, float* out) {
    Tex a(w, h, 4), b(w, h, 4);
    std::copy(in, in + size_t(w) * h * 4, a.f.begin());
    Matrix3x3 m;
    for (int r = 0; r < 3; r++) m.m[r] = metal::float3(m9[3 * r], m9[3 * r + 1], m9[3 * r + 2]);
    auto ta = a.t<float>();
    auto tb = b.t<float, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { transformImage(ta, tb, m, i); });
    std::copy(b.f.begin(), b.f.end(), out);
    return 0;
}

// despeckleLumaMedianChromaImage with the level-0 YCbCr NLF (raw_converter.cpp:76-78)
int ref_despeckle(const float* ycc, int w, int h, const gls_demosaic_params* p, float* out) {
    Tex a(w, h, 4), b(w, h, 4);
    std::copy(ycc, ycc + size_t(w) * h * 4, a.f.begin());
    metal::float3 va(p->pyramid_nlf[0].a[0], p->pyramid_nlf[0].a[1], p->pyramid_nlf[0].a[2]);
    metal::float3 vb(p->pyramid_nlf[0].b[0], p->pyramid_nlf[0].b[1], p->pyramid_nlf[0].b[2]);
    auto ta = a.t<half>();
    auto tb = b.t<half, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { despeckleLumaMedianChromaImage(ta, va, vb, tb, i); });
    std::copy(b.f.begin(), b.f.end(), out);
    return 0;
}

// PyramidProcessor<levels>::denoise, pyramid_processor.cpp:96-172, on a
// YCbCr image and its gradient. den_levels (optional) receives the denoised
// levels packed one after the other; bases (optional) the PCA bases used.
int ref_pyramid_denoise(const float* ycc, const float* grad, int w, int h, const gls_demosaic_params* p, float* out,
                        float* den_levels, double* bases) {
    const int L = p->levels;
    std::vector<Tex*> img(L), grd(L), sub(L), den(L), pca(L);
    for (int i = 0; i < L; i++) {
        const int wi = w >> i, hi = h >> i;
        img[i] = new Tex(wi, hi, 4);
        grd[i] = new Tex(wi, hi, 2);
        sub[i] = new Tex(wi, hi, 4);
        den[i] = new Tex(wi, hi, 4);
        pca[i] = new Tex(wi, hi, 4, metal::tex_fmt::u32);
    }
    std::copy(ycc, ycc + size_t(w) * h * 4, img[0]->f.begin());
    std::copy(grad, grad + size_t(w) * h * 2, grd[0]->f.begin());
    for (int i = 0; i < L - 1; i++) {  // :103-120
        auto a = img[i]->t<float>();
        auto b = img[i + 1]->t<float, access::write>();
        run_grid(img[i + 1]->st.width, img[i + 1]->st.height, [&](metal::uint2 x) { downsampleImageXYZ(a, b, x); });
        auto c = grd[i]->t<float>();
        auto d = grd[i + 1]->t<float, access::write>();
        run_grid(grd[i + 1]->st.width, grd[i + 1]->st.height, [&](metal::uint2 x) { downsampleImageXY(c, d, x); });
    }
    std::vector<metal::array<float, 25>> patches(size_t(w) * h / 64 + 1);
    for (int i = L - 1; i >= 0; i--) {  // :123-168
        const gls_denoise_params& dp = p->denoise[i];
        const int wi = w >> i, hi = h >> i;
        Tex* layer = img[i];
        if (i < L - 1) {
            float lw = 1.0f, sharp = dp.sharpening;
            metal::float2 nlf = f2(p->pyramid_nlf[i].a[0] * dp.luma, p->pyramid_nlf[i].b[0] * dp.luma);
            auto t0 = img[i]->t<float>();
            auto t1 = img[i + 1]->t<float>();
            auto t2 = den[i + 1]->t<float>();
            auto t3 = grd[i]->t<float>();
            auto to = sub[i]->t<float, access::write>();
            run_grid(wi, hi, [&](metal::uint2 x) { subtractNoiseImage(t0, t1, t2, t3, lw, sharp, nlf, to, x); });
            layer = sub[i];
        }
        // collectPatches on the reference's grid and indexing; the basis is
        // built from the dense (W/8) x (H/8) grid of written patches
        auto tl = layer->t<half>();
        const int gw = wi / 8, gh = hi / 8;
        std::fill(patches.begin(), patches.end(), metal::array<float, 25>{});
        run_grid(gw, gh, [&](metal::uint2 x) { collectPatches(tl, patches.data(), x); });
        std::array<std::array<double, 8>, 25> basis;
        {
            orc::Plane4<double> dense;  // rebuild an image whose 8-grid patches are the collected ones
            const int n = gw * gh;
            std::vector<double> pts(size_t(n) * 25);
            for (int y = 0; y < gh; y++)
                for (int x = 0; x < gw; x++) {
                    const int idx = y * wi / 8 + x;  // demosaic.metal:768
                    for (int k = 0; k < 25; k++) pts[size_t(y * gw + x) * 25 + k] = patches[idx][k];
                }
            if (n < 2) {
                for (int r = 0; r < 25; r++)
                    for (int c = 0; c < 8; c++) basis[r][c] = r == c ? 1.0 : 0.0;
            } else {
                double mean[25] = {0};
                for (int k = 0; k < n; k++)
                    for (int r = 0; r < 25; r++) mean[r] += pts[size_t(k) * 25 + r];
                for (int r = 0; r < 25; r++) mean[r] /= n;
                std::vector<double> cov(625, 0.0), vec;
                for (int k = 0; k < n; k++)
                    for (int r = 0; r < 25; r++)
                        for (int c = 0; c < 25; c++)
                            cov[r * 25 + c] += (pts[size_t(k) * 25 + r] - mean[r]) * (pts[size_t(k) * 25 + c] - mean[c]);
                for (auto& v : cov) v /= (n - 1);
                orc::jacobi_eigen(25, cov, vec);
                int idx[25];
                for (int k = 0; k < 25; k++) idx[k] = k;
                std::stable_sort(idx, idx + 25, [&](int a, int b) { return cov[a * 25 + a] > cov[b * 25 + b]; });
                double ev[25], evec[25][25];
                for (int c = 0; c < 25; c++) {
                    ev[c] = cov[idx[c] * 25 + idx[c]];
                    for (int r = 0; r < 25; r++) evec[r][c] = vec[r * 25 + idx[c]];
                }
                orc::select_basis(ev, evec, basis);
            }
        }
        if (bases)
            for (int r = 0; r < 25; r++)
                for (int c = 0; c < 8; c++) bases[(size_t(i) * 25 + r) * 8 + c] = basis[r][c];
        metal::array<metal::array<half, 8>, 25> space;
        for (int r = 0; r < 25; r++)
            for (int c = 0; c < 8; c++) space[r][c] = half(float(basis[r][c]));
        auto tp_w = pca[i]->t<uint, access::write>();
        run_grid(wi, hi, [&](metal::uint2 x) { pcaProjection(tl, &space, tp_w, x); });
        metal::float3 va(p->pyramid_nlf[i].a[0], p->pyramid_nlf[i].a[1], p->pyramid_nlf[i].a[2]);
        metal::float3 vb(p->pyramid_nlf[i].b[0], p->pyramid_nlf[i].b[1], p->pyramid_nlf[i].b[2]);
        metal::float3 tm(dp.luma, dp.chroma, dp.chroma);
        float cb = dp.chroma_boost, gb = dp.gradient_boost, gt = dp.gradient_threshold, lsc = p->lens_shading_correction;
        auto tg = grd[i]->t<half>();
        auto tp = pca[i]->t<uint>();
        auto td = den[i]->t<half, access::write>();
        run_grid(wi, hi, [&](metal::uint2 x) {
            blockMatchingDenoiseImage(tl, tg, tp, va, vb, tm, cb, gb, gt, lsc, td, x);
        });
    }
    std::copy(den[0]->f.begin(), den[0]->f.end(), out);
    if (den_levels) {
        size_t off = 0;
        for (int i = 0; i < L; i++) {
            std::copy(den[i]->f.begin(), den[i]->f.end(), den_levels + off);
            off += den[i]->f.size();
        }
    }
    for (int i = 0; i < L; i++) {
        delete img[i];
        delete grd[i];
        delete sub[i];
        delete den[i];
        delete pca[i];
    }
    return 0;
}

// RawConverter::demosaic (raw_converter.cpp:148-248, postProcess = false)
// end to end through the reference kernels: scale, Sobel + blur, the
// high-noise quad branch, demosaic + highlights, cam -> YCbCr, despeckle,
// the pyramid denoise and YCbCr -> cam. out: RGBA float (w = 0).
int ref_raw_pipeline(const uint16_t* raw, int w, int h, const gls_demosaic_params* p, int denoise, float* out) {
    const size_t n = size_t(w) * h;
    std::vector<float> scaled(n), grad(n * 2), rgb(n * 4), ycc(n * 4), desp(n * 4), den(n * 4);
    ref_scale(raw, w, h, p, scaled.data());
    ref_sobel_blur(scaled.data(), w, h, p, grad.data());
    if (denoise && p->high_noise_image) ref_raw_denoise(scaled.data(), grad.data(), w, h, p, scaled.data());
    ref_demosaic_rgb(scaled.data(), grad.data(), w, h, p, rgb.data());
    if (!denoise) {
        std::copy(rgb.begin(), rgb.end(), out);
        return 0;
    }
    const orc::Mat3 c2y = orc::cam_ycbcr(p->rgb_cam, p->xyz_rgb), y2c = orc::inverse3(c2y);
    ref_transform(rgb.data(), w, h, &c2y.m[0][0], ycc.data());
    ref_despeckle(ycc.data(), w, h, p, desp.data());
    ref_pyramid_denoise(desp.data(), grad.data(), w, h, p, den.data(), nullptr, nullptr);
    ref_transform(den.data(), w, h, &y2c.m[0][0], out);
    return 0;
}

int ref_noise_tables(unsigned seed, int* perm, float* grad);

// basicRawNoiseStatistics (demosaic.metal:1110-1136) over a scaled raw frame
// (RawConverter::MeasureRawNLF, raw_converter.cpp:340): 9x9 mean and
// variance of the four channels at every half-resolution position.
int ref_raw_noise_stats(const float* scaled, int w, int h, int pattern, float* mean, float* var) {
    Tex s(w, h, 1), m(w / 2, h / 2, 4), v(w / 2, h / 2, 4);
    std::copy(scaled, scaled + size_t(w) * h, s.f.begin());
    auto ts = s.t<float>();
    auto tm = m.t<float, access::write>();
    auto tv = v.t<float, access::write>();
    int bp = pattern;
    run_grid(w / 2, h / 2, [&](metal::uint2 i) { basicRawNoiseStatistics(ts, bp, tm, tv, i); });
    std::copy(m.f.begin(), m.f.end(), mean);
    std::copy(v.f.begin(), v.f.end(), var);
    return 0;
}

// basicNoiseStatistics (demosaic.metal:1138-1159) over one YCbCr pyramid
// level (PyramidProcessor::MeasureYCbCrNLF, pyramid_processor.cpp:180):
// 5x5 mean of Y and variances of Y, Cb, Cr.
int ref_ycc_noise_stats(const float* img, int w, int h, float* stats) {
    Tex in(w, h, 4), st(w, h, 4);
    std::copy(img, img + size_t(w) * h * 4, in.f.begin());
    auto ti = in.t<float>();
    auto ts = st.t<float, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { basicNoiseStatistics(ti, ts, i); });
    std::copy(st.f.begin(), st.f.end(), stats);
    return 0;
}

// RawConverter::demosaic's post-processing (raw_converter.cpp:87-112 and
// 231-241): the histogram of denoised level 3 and its statistics, the
// guided-filter (a, b) of levels 4, 2 and 0 with their box filter, the
// tone-mapping mask at full size, and convertTosRGB with the grain seeded by
// `seed`. den_levels: the 5 denoised levels (YCbCr RGBA float, packed level
// after level), or NULL for a frame without noise reduction (the fixed
// statistics of raw_converter.cpp:225-229; the reference computes no mask
// then, so local tone mapping must be off: returns 2 otherwise).
// grad: the level-0 gradient (2 floats per pixel); rgb: the linear camera
// RGB (RGBA float). out: RGBA float; stats: black, white, shadows,
// highlights, mean, median.
int ref_postprocess(const float* den_levels, const float* grad, const float* rgb, int w, int h,
                    const gls_demosaic_params* p, unsigned seed, float* out, float* stats) {
    const gls_rgb_conversion_params& rc = p->rgb_conversion;
    if (!den_levels && rc.local_tone_mapping) return 2;
    histogram_data hd{};
    Tex mask(w, h, 1);
    std::vector<Tex*> den;
    if (den_levels) {
        size_t off = 0;
        for (int l = 0; l < 5; l++) {
            const int wl = w >> l, hl = h >> l;
            Tex* t = new Tex(wl, hl, 4);
            std::copy(den_levels + off, den_levels + off + size_t(wl) * hl * 4, t->f.begin());
            off += size_t(wl) * hl * 4;
            den.push_back(t);
        }
        // raw_converter.cpp:87-90
        auto t3 = den[3]->t<float>();
        run_grid(w >> 3, h >> 3, [&](metal::uint2 i) { histogramImage(t3, hd, i); });
        const metal::uint2 dims(uint(w >> 3), uint(h >> 3));
        histogramStatistics(hd, dims, metal::uint2(0u, 0u));
    } else {
        hd.black_level = 0.1f;
        hd.white_level = 1.0f;
        hd.mean = 0.22f;
        hd.median = 0.22f;
    }
    if (den_levels && rc.local_tone_mapping) {
        // LocalToneMapping::createMask (raw_converter.hpp:61-75), guides =
        // denoised levels 4, 2, 0 (raw_converter.cpp:105-112)
        LTMParameters lp;
        lp.eps = p->ltm.eps;
        lp.shadows = p->ltm.shadows;
        lp.highlights = p->ltm.highlights;
        for (int k = 0; k < 3; k++) lp.detail[k] = p->ltm.detail[k];
        std::vector<Tex*> abm;
        for (int k : {4, 2, 0}) {
            const int wk = w >> k, hk = h >> k;
            Tex ab(wk, hk, 2);
            Tex* mean = new Tex(wk, hk, 2);
            auto tg = den[k]->t<float>();
            auto tab_w = ab.t<float, access::write>();
            const float eps = lp.eps;
            run_grid(wk, hk, [&](metal::uint2 i) { GuidedFilterABImage(tg, tab_w, eps, i); });
            auto tab = ab.t<float>();
            auto tm_w = mean->t<float, access::write>();
            run_grid(wk, hk, [&](metal::uint2 i) { BoxFilterGFImage(tab, tm_w, i); });
            abm.push_back(mean);
        }
        Tex g(w, h, 2);
        std::copy(grad, grad + size_t(w) * h * 2, g.f.begin());
        const metal::float2 nlf = f2(p->pyramid_nlf[0].a[0], p->pyramid_nlf[0].b[0]);
        auto t0 = den[0]->t<float>();
        auto tg = g.t<float>();
        auto lf = abm[0]->t<float>(), mf = abm[1]->t<float>(), hf = abm[2]->t<float>();
        auto tmask_w = mask.t<float, access::write>();
        run_grid(w, h, [&](metal::uint2 i) {
            localToneMappingMaskImage(t0, tg, lf, mf, hf, tmask_w, lp, nlf, hd, i);
        });
        for (Tex* t : abm) delete t;
    }
    // convertTosRGB (demosaic_kernels.hpp:629-671, raw_converter.cpp:231-241)
    RGBConversionParameters cp;
    cp.contrast = rc.contrast;
    cp.saturation = rc.saturation;
    cp.toneCurveSlope = rc.tone_curve_slope;
    cp.exposureBias = rc.exposure_bias;
    cp.exposureBias += std::log2(p->exposure_multiplier);
    cp.blacks = rc.blacks;
    cp.localToneMapping = rc.local_tone_mapping != 0;
    Matrix3x3 tr;
    for (int r = 0; r < 3; r++) tr.m[r] = metal::float3(p->rgb_cam[3 * r], p->rgb_cam[3 * r + 1], p->rgb_cam[3 * r + 2]);
    const metal::float2 luma_var = f2(2.0f * ((p->raw_nlf.a[1] + p->raw_nlf.a[3]) / 2),
                                      2.0f * ((p->raw_nlf.b[1] + p->raw_nlf.b[3]) / 2));
    metal::array<int, 514> perm;
    metal::array<metal::float2, 514> g2;
    {
        float gt[514 * 2];
        ref_noise_tables(seed, perm.data(), gt);
        for (int i = 0; i < 514; i++) g2[i] = f2(gt[2 * i], gt[2 * i + 1]);
    }
    Tex lin(w, h, 4), o(w, h, 4);
    std::copy(rgb, rgb + size_t(w) * h * 4, lin.f.begin());
    auto tl = lin.t<float>();
    auto tmask = mask.t<float>();
    auto to_w = o.t<float, access::write>();
    run_grid(w, h, [&](metal::uint2 i) { convertTosRGB(tl, tmask, to_w, tr, cp, hd, luma_var, perm, g2, i); });
    std::copy(o.f.begin(), o.f.end(), out);
    if (stats) {
        const float v[6] = {hd.black_level, hd.white_level, hd.shadows, hd.highlights, hd.mean, hd.median};
        std::copy(v, v + 6, stats);
    }
    for (Tex* t : den) delete t;
    return 0;
}

// RawConverter::demosaic(postProcess = true) end to end through the
// reference kernels: ref_raw_pipeline's stages, keeping the five denoised
// levels, then ref_postprocess seeded with the first raw pixel
// (raw_converter.cpp:238). Noise reduction needs levels == 5.
int ref_demosaic_post(const uint16_t* raw, int w, int h, const gls_demosaic_params* p, int denoise, float* out,
                      float* stats) {
    const size_t n = size_t(w) * h;
    std::vector<float> scaled(n), grad(n * 2), rgb(n * 4), ycc(n * 4), desp(n * 4), den(n * 4), cam(n * 4);
    std::vector<float> levels;
    ref_scale(raw, w, h, p, scaled.data());
    ref_sobel_blur(scaled.data(), w, h, p, grad.data());
    if (denoise && p->high_noise_image) ref_raw_denoise(scaled.data(), grad.data(), w, h, p, scaled.data());
    ref_demosaic_rgb(scaled.data(), grad.data(), w, h, p, rgb.data());
    if (!denoise) return ref_postprocess(nullptr, grad.data(), rgb.data(), w, h, p, raw[0], out, stats);
    if (p->levels != 5) return 3;
    size_t tot = 0;
    for (int l = 0; l < 5; l++) tot += size_t(w >> l) * (h >> l) * 4;
    levels.resize(tot);
    const orc::Mat3 c2y = orc::cam_ycbcr(p->rgb_cam, p->xyz_rgb), y2c = orc::inverse3(c2y);
    ref_transform(rgb.data(), w, h, &c2y.m[0][0], ycc.data());
    ref_despeckle(ycc.data(), w, h, p, desp.data());
    ref_pyramid_denoise(desp.data(), grad.data(), w, h, p, den.data(), levels.data(), nullptr);
    ref_transform(den.data(), w, h, &y2c.m[0][0], cam.data());
    return ref_postprocess(levels.data(), grad.data(), cam.data(), w, h, p, raw[0], out, stats);
}

// convertToGrayscale (demosaic.metal:1707-1723): rgb w x h x 4, gray w x h
int ref_convert_to_grayscale(const float* rgb, int w, int h, const float* t, float* gray) {
    Tex in(w, h, 4), out(w, h, 1);
    std::copy(rgb, rgb + size_t(w) * h * 4, in.f.begin());
    auto ti = in.t<float>();
    auto to = out.t<float, access::write>();
    const metal::float3 tr(t[0], t[1], t[2]);
    run_grid(w, h, [&](metal::uint2 i) { convertToGrayscale(ti, to, tr, i); });
    std::copy(out.f.begin(), out.f.end(), gray);
    return 0;
}

void ref_set_threads(int n) { orc::num_threads() = n > 0 ? n : 1; }

}  // extern "C"
