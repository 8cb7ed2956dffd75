// ref_nlf.cpp — TEST INFRASTRUCTURE ONLY. The reference's own noise-model
// regressions compiled for the CPU as the pin of the oracle's restatement
// (oracle/gls_oracle_nlf.hpp):
//   * RawConverter::MeasureRawNLF     MetalPipeline/raw_converter.cpp:339-490
//   * PyramidProcessor<5>::MeasureYCbCrNLF
//                                     MetalPipeline/pyramid_processor.cpp:173-324
// The recipe (oracle/Makefile, target ref) extracts those unmodified line
// ranges into _ref/. This file supplies what they touch: the GlassImage
// vector and image types (gls_shim/gls_nlf.hpp), the Metal context, and
// class shells with the members the two functions use. The statistics
// kernels they launch are no-ops here: the caller fills the statistics
// images (with the reference's basicRawNoiseStatistics /
// basicNoiseStatistics kernels, ref_harness.cpp). Part of
// _ref/libglsref.so.
#include <algorithm>
#include <cassert>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <memory>
#include <utility>

#include "gls_nlf.hpp"

using std::max;

// The two functions report their fits on std::cout. This library carries
// its own static copy of the C++ runtime, whose standard streams are not
// set up when a host process (Python) loads it, so the reports go to a
// sink that discards them; nothing they compute reads the stream.
namespace nlf_log {
struct Sink {
    template <class T>
    Sink& operator<<(const T&) {
        return *this;
    }
    Sink& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
inline Sink sink;
}  // namespace nlf_log
namespace std {
using nlf_log::sink;
}
#define cout sink

struct MetalContext {
    void waitForCompletion() {}
};

enum BayerPattern { grbg = 0, gbrg = 1, rggb = 2, bggr = 3 };

typedef std::pair<gls::Vector<4>, gls::Vector<4>> RawNLF;    // demosaic.hpp:51
typedef std::pair<gls::Vector<3>, gls::Vector<3>> YCbCrNLF;  // demosaic.hpp:53

class RawConverter {
   public:
    struct RawStats {
        void operator()(MetalContext*, const gls::mtl_image_2d<gls::pixel_float>&, int,
                        gls::mtl_image_2d<gls::pixel_float4>*, gls::mtl_image_2d<gls::pixel_float4>*) const {}
    };
    MetalContext _mtlContext;
    RawStats _rawNoiseStatistics;
    std::unique_ptr<gls::mtl_image_2d<gls::luma_pixel_16>> _rawImage;
    std::unique_ptr<gls::mtl_image_2d<gls::pixel_float>> _scaledRawImage;
    std::unique_ptr<gls::mtl_image_2d<gls::pixel_float4>> _meanImage, _varImage;

    RawNLF MeasureRawNLF(float exposure_multiplier, BayerPattern bayerPattern);
};

using namespace gls;

#include "measure_raw_nlf.inc"

template <size_t levels>
class PyramidProcessor {
   public:
    struct Stats {
        void operator()(MetalContext*, const gls::mtl_image_2d<gls::pixel_float4>&,
                        gls::mtl_image_2d<gls::pixel_float4>*) const {}
    };
    Stats _basicNoiseStatistics;

    YCbCrNLF MeasureYCbCrNLF(MetalContext* context, const gls::mtl_image_2d<gls::pixel_float4>& inputImage,
                             gls::mtl_image_2d<gls::pixel_float4>* noiseStats, float exposure_multiplier);
};

#include "measure_ycc_nlf.inc"

template class PyramidProcessor<5>;

namespace {
void fill4(gls::mtl_image_2d<gls::pixel_float4>& img, const float* src) {
    for (size_t i = 0; i < img.px.size(); i++)
        for (int c = 0; c < 4; c++) img.px[i].v[size_t(c)] = src[4 * i + size_t(c)];
}
}  // namespace

extern "C" {

// MeasureRawNLF over the 9x9 statistics of a raw frame: mean and var are the
// (raw_w / 2) x (raw_h / 2) RGBA float images basicRawNoiseStatistics wrote.
// a, b: the four channels' variance model. Returns 2, without running the
// reference code, if a first-channel variance is negative: the reference
// then converts a NaN logarithm to an int and indexes its histogram with it
// (raw_converter.cpp:362), which is undefined.
int ref_measure_raw_nlf(const float* mean, const float* var, int raw_w, int raw_h, float exposure_multiplier,
                        float* a, float* b) {
    const size_t n = size_t(raw_w / 2) * size_t(raw_h / 2);
    for (size_t i = 0; i < n; i++)
        if (var[4 * i] < 0.f) return 2;
    RawConverter rc;
    rc._rawImage = std::make_unique<gls::mtl_image_2d<gls::luma_pixel_16>>(raw_w, raw_h);
    rc._meanImage = std::make_unique<gls::mtl_image_2d<gls::pixel_float4>>(raw_w / 2, raw_h / 2);
    rc._varImage = std::make_unique<gls::mtl_image_2d<gls::pixel_float4>>(raw_w / 2, raw_h / 2);
    rc._scaledRawImage = std::make_unique<gls::mtl_image_2d<gls::pixel_float>>(1, 1);
    fill4(*rc._meanImage, mean);
    fill4(*rc._varImage, var);
    const RawNLF nlf = rc.MeasureRawNLF(exposure_multiplier, rggb);
    for (int c = 0; c < 4; c++) {
        a[c] = nlf.first[size_t(c)];
        b[c] = nlf.second[size_t(c)];
    }
    return 0;
}

// MeasureYCbCrNLF over the 5x5 statistics of one pyramid level: stats is the
// w x h RGBA float image basicNoiseStatistics wrote (mean Y, var Y, Cb, Cr).
int ref_measure_ycc_nlf(const float* stats, int w, int h, float exposure_multiplier, float* a, float* b) {
    PyramidProcessor<5> pp;
    MetalContext ctx;
    gls::mtl_image_2d<gls::pixel_float4> input(w, h), noise_stats(w, h);
    fill4(noise_stats, stats);
    const YCbCrNLF nlf = pp.MeasureYCbCrNLF(&ctx, input, &noise_stats, exposure_multiplier);
    for (int c = 0; c < 3; c++) {
        a[c] = nlf.first[size_t(c)];
        b[c] = nlf.second[size_t(c)];
    }
    return 0;
}

}  // extern "C"
