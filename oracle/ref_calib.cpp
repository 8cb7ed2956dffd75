// ref_calib.cpp — TEST INFRASTRUCTURE ONLY. The reference's own camera
// calibration compiled for the CPU, so that the reference arm of the bench
// and the pin tests take their DemosaicParameters from the reference's code
// rather than from the library under test:
//   * the parameter types       MetalPipeline/demosaic.hpp:29-60, 95-124
//   * the NLF and smoothstep helpers            demosaic.hpp:154-184
//   * iPhone14WideCalibration (nlfFromIso, getDenoiseParameters,
//     buildDemosaicParameters)   MetalPipeline/iPhone14WideCalibration.cpp:28-138
//   * its NLF table                             iPhone14WideCalibration.cpp:151-252
// The recipe (oracle/Makefile, target ref) extracts those unmodified line
// ranges into _ref/. This file supplies what they touch: the GlassImage
// Vector / Matrix stand-ins (gls_shim/gls_linalg.hpp), a CameraCalibration
// shell with the three virtual members, and the assembly of
// CameraCalibration::getDemosaicParameters (CameraCalibration.cpp:39-54)
// for a given ISO. Part of _ref/libglsref.so.
#include <algorithm>
#include <array>
#include <cmath>
#include <iostream>
#include <string>
#include <utility>

#include "../include/glscam.h"
#include "gls_linalg.hpp"

// getDenoiseParameters reports on std::cout; the report goes to a sink
// (this library's copy of the C++ runtime has no standard streams set up
// when a Python process loads it), nothing computed reads it.
namespace calib_log {
struct Sink {
    template <class T>
    Sink& operator<<(const T&) {
        return *this;
    }
    Sink& operator<<(std::ostream& (*)(std::ostream&)) { return *this; }
};
inline Sink sink;
}  // namespace calib_log
namespace std {
using calib_log::sink;
}
#define cout sink

enum BayerPattern { grbg = 0, gbrg = 1, rggb = 2, bggr = 3 };  // demosaic.hpp:25

#include "calib_types.inc"
#include "calib_params.inc"
#include "calib_lerp.inc"

template <size_t levels = 5>
class CameraCalibration {  // CameraCalibration.hpp:24-31, the virtual members
   public:
    virtual ~CameraCalibration() {}
    virtual NoiseModel<levels> nlfFromIso(int iso) const = 0;
    virtual std::pair<RAWDenoiseParameters, std::array<DenoiseParameters, levels>> getDenoiseParameters(
        int iso) const = 0;
    virtual DemosaicParameters buildDemosaicParameters() const = 0;
};

#include "calib_iphone14wide.inc"
#include "calib_iphone14wide_nlf.inc"

#undef cout

extern "C" int ref_calibration_fill(int iso, gls_demosaic_params* p) {
    if (!p) return 1;
    iPhone14WideCalibration<5> cal;
    DemosaicParameters dp;
    try {
        // CameraCalibration::getDemosaicParameters, CameraCalibration.cpp:39-54
        // (the DNG-metadata part, unpackDNGMetadata, is the caller's)
        dp = cal.buildDemosaicParameters();
        const auto nlf = cal.nlfFromIso(iso);
        const auto den = cal.getDenoiseParameters(iso);
        dp.noiseModel = nlf;
        dp.rawDenoiseParameters = den.first;
        dp.denoiseParameters = den.second;
        dp.iso = iso;
    } catch (const std::exception&) {
        return 7;  // std::range_error on an ISO outside the table
    }
    for (int c = 0; c < 4; c++) {
        p->raw_nlf.a[c] = dp.noiseModel.rawNlf.first[c];
        p->raw_nlf.b[c] = dp.noiseModel.rawNlf.second[c];
    }
    for (int l = 0; l < 5; l++) {
        for (int c = 0; c < 3; c++) {
            p->pyramid_nlf[l].a[c] = dp.noiseModel.pyramidNlf[l].first[c];
            p->pyramid_nlf[l].b[c] = dp.noiseModel.pyramidNlf[l].second[c];
        }
        const DenoiseParameters& d = dp.denoiseParameters[l];
        p->denoise[l] = {d.luma, d.chroma, d.chromaBoost, d.gradientBoost, d.gradientThreshold, d.sharpening};
    }
    p->high_noise_image = dp.rawDenoiseParameters.highNoiseImage ? 1 : 0;
    p->raw_denoise_strength = dp.rawDenoiseParameters.strength;
    p->iso = dp.iso;
    p->lens_shading_correction = dp.lensShadingCorrection;
    const RGBConversionParameters& r = dp.rgbConversionParameters;
    p->rgb_conversion = {r.contrast, r.saturation, r.toneCurveSlope, r.exposureBias, r.blacks,
                         r.localToneMapping ? 1 : 0};
    const LTMParameters& t = dp.ltmParameters;
    p->ltm = {t.eps, t.shadows, t.highlights, {t.detail[0], t.detail[1], t.detail[2]}};
    return 0;
}
