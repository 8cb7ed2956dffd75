/*
 * glscam.hpp — header-only C++ facade over the C ABI of glscam.h, with the
 * class and method names of the reference's C++ API, so that a caller of
 * GlassCameraPublic's RawConverter / PyramidProcessor / CameraCalibration /
 * SURF / FindHomography / RegisterAndFuseKernel switches by changing types
 * and includes:
 *
 *   RawConverter            MetalPipeline/raw_converter.hpp:80-188
 *   PyramidProcessor        MetalPipeline/pyramid_processor.hpp:23-76
 *   CameraCalibration       MetalPipeline/CameraCalibration.hpp:24-39,
 *   iPhone14WideCalibration MetalPipeline/iPhone14WideCalibration.cpp
 *   SURF, DMatch, KeyPoint  ImageRegistration/SURF.hpp:29-80, feature2d.hpp:25-47
 *   FindHomography,         ImageRegistration/Homography.hpp:26-37
 *   ScaleHomography
 *   RegisterAndFuseKernel   MetalPipeline/demosaic_kernels.hpp:690-710
 *   RawChannels             PyramidFusion/pyramidFusion.cpp:106-143
 *
 * Differences a caller sees:
 *   * images are device pointers (CUDA) instead of Metal textures; host
 *     pointers are accepted where the C ABI takes GLS_HOST_IO;
 *   * errors: the C ABI returns status codes; this facade throws
 *     std::range_error for GLS_ERR_RANGE and GLS_ERR_DEGENERATE (where the
 *     reference throws it: iPhone14WideCalibration.cpp:61,
 *     LeastSquaresHomography.cpp:383) and std::runtime_error otherwise;
 *   * calls run on a CUDA stream; the methods that return host data
 *     synchronise, as the reference's waitForCompletion() does.
 *
 * Link with libglscam.so (glasscamerapublic_b200/libglscam.so).
 */
#ifndef GLSCAM_HPP
#define GLSCAM_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "glscam.h"

namespace gls {

inline void check(gls_status s) {
    if (s == GLS_OK) return;
    const std::string msg = std::string("glscam: ") + gls_last_error_message();
    if (s == GLS_ERR_RANGE || s == GLS_ERR_DEGENERATE) throw std::range_error(msg);
    throw std::runtime_error(msg);
}

constexpr uint32_t flag_if(bool on, uint32_t f) { return on ? f : 0u; }

using DemosaicParameters = gls_demosaic_params;
using ImageView = gls_image_view;

enum BayerPattern { grbg = GLS_GRBG, gbrg = GLS_GBRG, rggb = GLS_RGGB, bggr = GLS_BGGR };

// ---------------------------------------------------------------- calibration
template <size_t levels = 5>
class CameraCalibration {
   public:
    explicit CameraCalibration(int32_t camera) : camera_(camera) {}
    virtual ~CameraCalibration() = default;

    // nlfFromIso + getDenoiseParameters into a parameter block
    DemosaicParameters getDemosaicParameters(int iso) const {
        DemosaicParameters p{};
        p.levels = int32_t(levels);
        check(gls_calibration_fill(camera_, iso, &p));
        p.levels = int32_t(levels);
        return p;
    }
    // getDemosaicParameters(raw, xyz_rgb, &dng_metadata, &exif_metadata)
    // (CameraCalibration.cpp:25-58) from a DNG's metadata (read_dng_file)
    DemosaicParameters getDemosaicParameters(const gls_dng_info& dng, const float* xyz_rgb = nullptr) const {
        DemosaicParameters p{};
        check(gls_dng_demosaic_params(&dng, xyz_rgb, camera_, &p));
        p.levels = int32_t(levels);
        return p;
    }
    std::pair<gls_raw_nlf, std::array<gls_ycbcr_nlf, levels>> nlfFromIso(int iso) const {
        const DemosaicParameters p = getDemosaicParameters(iso);
        std::array<gls_ycbcr_nlf, levels> y{};
        for (size_t i = 0; i < levels; i++) y[i] = p.pyramid_nlf[i];
        return {p.raw_nlf, y};
    }
    std::array<gls_denoise_params, levels> getDenoiseParameters(int iso) const {
        const DemosaicParameters p = getDemosaicParameters(iso);
        std::array<gls_denoise_params, levels> d{};
        for (size_t i = 0; i < levels; i++) d[i] = p.denoise[i];
        return d;
    }

   private:
    int32_t camera_;
};

template <size_t levels = 5>
class iPhone14WideCalibration : public CameraCalibration<levels> {
   public:
    iPhone14WideCalibration() : CameraCalibration<levels>(GLS_CAMERA_IPHONE14_WIDE) {}
};

// ---------------------------------------------------------------- RawConverter
class RawConverter {
   public:
    // RawConverter(device, icc, calibrateFromImage) (raw_converter.hpp:128-156)
    explicit RawConverter(int device = 0, const std::vector<uint8_t>* icc = nullptr,
                          bool calibrateFromImage = false) {
        check(gls_converter_create(device, icc ? icc->data() : nullptr, icc ? icc->size() : 0,
                                   calibrateFromImage ? 1 : 0, &conv_));
    }
    ~RawConverter() { gls_converter_destroy(conv_); }
    RawConverter(const RawConverter&) = delete;
    RawConverter& operator=(const RawConverter&) = delete;

    // demosaic(raw, params, noiseReduction, postProcess) (raw_converter.hpp:182-183):
    // the result is a view of converter-owned device memory (RGBA), valid
    // until the next call, as the reference's returned texture is. raw is
    // device memory, or host memory with host_input.
    ImageView demosaic(const uint16_t* raw, int width, int height, size_t stride_bytes,
                       const DemosaicParameters* params, bool noiseReduction = true, bool postProcess = false,
                       bool fp16 = false, bool host_input = false, void* stream = nullptr) {
        ImageView out{};
        uint32_t flags = flag_if(noiseReduction, GLS_DENOISE) | flag_if(postProcess, GLS_POSTPROCESS) |
                         flag_if(fp16, GLS_FP16_STORAGE) | flag_if(host_input, GLS_HOST_IO) | uint32_t(GLS_SYNC);
        check(gls_demosaic(conv_, raw, width, height, stride_bytes, params, flags, &out, stream));
        return out;
    }

    // demosaic into a caller buffer (F32 or F16 RGBA, device memory, or host
    // memory with host_io), asynchronous on the stream unless host_io
    void demosaic(const uint16_t* raw, int width, int height, size_t stride_bytes, const DemosaicParameters* params,
                  ImageView* out, bool noiseReduction = true, bool fp16 = true, bool host_io = false,
                  void* stream = nullptr, bool postProcess = false) {
        uint32_t flags = flag_if(noiseReduction, GLS_DENOISE) | flag_if(fp16, GLS_FP16_STORAGE) |
                         flag_if(host_io, GLS_HOST_IO) | flag_if(postProcess, GLS_POSTPROCESS);
        check(gls_demosaic(conv_, raw, width, height, stride_bytes, params, flags, out, stream));
    }

    // MeasureRawNLF (raw_converter.cpp:339-490) on a scaled raw frame
    // (1 ch F32/F16 device memory); synchronous
    gls_raw_nlf MeasureRawNLF(const ImageView& scaled, BayerPattern pattern, float exposure_multiplier = 1,
                              void* stream = nullptr) {
        gls_raw_nlf n{};
        check(gls_measure_raw_nlf(conv_, &scaled, int32_t(pattern), exposure_multiplier, &n, stream));
        return n;
    }

    // the models the last call of a calibrateFromImage converter measured
    std::pair<gls_raw_nlf, std::vector<gls_ycbcr_nlf>> noiseModel() const {
        gls_raw_nlf r{};
        std::vector<gls_ycbcr_nlf> y(GLS_MAX_LEVELS);
        int32_t n = 0;
        check(gls_converter_noise_model(conv_, &r, y.data(), GLS_MAX_LEVELS, &n));
        y.resize(size_t(n));
        return {r, y};
    }

    // many frames of any sizes in one call (no reference counterpart); graph
    // records the batch and replays it while frames, buffers and
    // parameters stay the same
    void demosaic_batch(std::vector<gls_frame_desc>& frames, bool noiseReduction = true, bool fp16 = true,
                        bool host_io = false, void* stream = nullptr, bool graph = false) {
        uint32_t flags = flag_if(noiseReduction, GLS_DENOISE) | flag_if(fp16, GLS_FP16_STORAGE) |
                         flag_if(host_io, GLS_HOST_IO) | flag_if(graph, GLS_GRAPH);
        check(gls_demosaic_batch(conv_, frames.data(), int32_t(frames.size()), flags, stream));
    }

    // calibration gradient (no reference counterpart): the MSE of the FP32
    // path's RGB against target (F32 RGB or RGBA) and its gradient with
    // respect to the GLS_ADJ_NPARAMS parameters (gls_demosaic_denoise_vjp)
    double demosaic_denoise_vjp(const uint16_t* raw, int width, int height, size_t stride_bytes,
                                const DemosaicParameters* params, const ImageView& target,
                                std::array<float, GLS_ADJ_NPARAMS>* grad, bool host_io = false,
                                void* stream = nullptr) {
        double loss = 0;
        check(gls_demosaic_denoise_vjp(conv_, raw, width, height, stride_bytes, params, &target,
                                       flag_if(host_io, GLS_HOST_IO), &loss, grad->data(), stream));
        return loss;
    }

    gls_converter* handle() const { return conv_; }

   private:
    gls_converter* conv_ = nullptr;
};

// ---------------------------------------------------------------- PyramidProcessor
template <size_t levels = 5>
class PyramidProcessor {
   public:
    explicit PyramidProcessor(RawConverter& converter) : conv_(converter.handle()) {}

    // denoise(ycc, gradient, params) (pyramid_processor.hpp:59-62): YCbCr
    // (4 ch) and gradient (2 ch) in, denoised YCbCr out
    void denoise(const ImageView& ycc, const ImageView& gradient, const DemosaicParameters* params, ImageView* out,
                 bool fp16 = false, bool host_io = false, void* stream = nullptr) {
        DemosaicParameters p = *params;
        p.levels = int32_t(levels);
        uint32_t flags = flag_if(fp16, GLS_FP16_STORAGE) | flag_if(host_io, GLS_HOST_IO | GLS_SYNC);
        check(gls_pyramid_denoise(conv_, &ycc, &gradient, &p, flags, out, stream));
    }

    // the denoise's vector-Jacobian product (gls_pyramid_denoise_vjp):
    // g_out = dL/d(denoised YCbCr) in; dL/dtheta and, if g_ycc is given,
    // dL/d(ycc) out
    void denoise_vjp(const ImageView& ycc, const ImageView& gradient, const DemosaicParameters* params,
                     const ImageView& g_out, std::array<float, GLS_ADJ_NPARAMS>* grad, ImageView* g_ycc = nullptr,
                     bool host_io = false, void* stream = nullptr) {
        DemosaicParameters p = *params;
        p.levels = int32_t(levels);
        check(gls_pyramid_denoise_vjp(conv_, &ycc, &gradient, &p, &g_out, flag_if(host_io, GLS_HOST_IO), grad->data(),
                                      g_ycc, stream));
    }

    // MeasureYCbCrNLF (pyramid_processor.cpp:173-324) on a YCbCr image
    // (4 ch F32/F16 device memory); synchronous
    gls_ycbcr_nlf MeasureYCbCrNLF(const ImageView& image, float exposure_multiplier = 1, void* stream = nullptr) {
        gls_ycbcr_nlf n{};
        check(gls_measure_ycbcr_nlf(conv_, &image, exposure_multiplier, &n, stream));
        return n;
    }

   private:
    gls_converter* conv_;
};

// ---------------------------------------------------------------- registration
using KeyPoint = gls_keypoint;
using DMatch = gls_match;

struct Point2f {
    float x = 0, y = 0;
};

class SURF {
   public:
    // SURF::makeInstance (SURF.hpp:45-47)
    static SURF makeInstance(int width, int height, int max_features = -1, int nOctaves = 4, int nOctaveLayers = 2,
                             float hessianThreshold = 0.02f, int device = 0) {
        return SURF(width, height, max_features, nOctaves, nOctaveLayers, hessianThreshold, device);
    }
    SURF(int width, int height, int max_features = -1, int nOctaves = 4, int nOctaveLayers = 2,
         float hessianThreshold = 0.02f, int device = 0)
        : max_features_(max_features) {
        check(gls_surf_create(device, width, height, max_features, nOctaves, nOctaveLayers, hessianThreshold, &s_));
    }
    SURF(SURF&& o) noexcept : s_(o.s_), max_features_(o.max_features_), next_(o.next_), detect_flags_(o.detect_flags_) {
        o.s_ = nullptr;
    }
    SURF(const SURF&) = delete;
    ~SURF() { gls_surf_destroy(s_); }

    // The reference's detector by default; true selects the corrected one
    // (per-axis maxima interpolation, every keypoint described:
    // GLS_SURF_CORRECTED).
    void setCorrectedDetector(bool on) { detect_flags_ = on ? uint32_t(GLS_SURF_CORRECTED) : 0u; }

    // detectAndCompute (SURF.hpp:57-58): img is a width x height float
    // image (device memory, or host memory with host_input); keypoints and
    // 64-float descriptors come back in host memory. The result also stays
    // in a feature slot of the detector (returned) for matchKeyPoints.
    int detectAndCompute(const float* img, int width, int height, size_t stride_bytes, std::vector<KeyPoint>* keypoints,
                         std::vector<float>* descriptors, bool host_input = false, void* stream = nullptr) {
        const int slot = next_;
        next_ = (next_ + 1) % GLS_SURF_SLOTS;
        ImageView v{const_cast<float*>(img), width, height, 1, GLS_F32, stride_bytes};
        check(gls_surf_detect_and_compute(s_, &v, slot,
                                          (host_input ? uint32_t(GLS_HOST_IO) : uint32_t(GLS_SYNC)) | detect_flags_,
                                          stream));
        const int cap = max_features_ >= 0 ? max_features_ : GLS_SURF_MAX_KEYPOINTS;
        keypoints->resize(size_t(cap));
        if (descriptors) descriptors->resize(size_t(cap) * 64);
        int32_t n = 0;
        check(gls_surf_features(s_, slot, keypoints->data(), descriptors ? descriptors->data() : nullptr, cap, &n,
                                stream));
        keypoints->resize(size_t(n));
        if (descriptors) descriptors->resize(size_t(n) * 64);
        return slot;
    }

    // Features that another detector computed (another GPU's
    // detectAndCompute, received by broadcast) into a slot of this one, for
    // matchKeyPoints; host memory. Returns the slot.
    int loadFeatures(const std::vector<KeyPoint>& keypoints, const std::vector<float>& descriptors) {
        if (descriptors.size() != keypoints.size() * 64)
            throw std::runtime_error("loadFeatures: 64 descriptor floats per keypoint");
        const int slot = next_;
        next_ = (next_ + 1) % GLS_SURF_SLOTS;
        check(gls_surf_load_features(s_, slot, keypoints.data(), descriptors.data(), int32_t(keypoints.size()),
                                     GLS_HOST_IO, nullptr));
        return slot;
    }

    // matchKeyPoints (SURF.cpp:931-974) between two detection slots
    std::vector<DMatch> matchKeyPoints(int query_slot, int train_slot, void* stream = nullptr) {
        const int cap = max_features_ >= 0 ? max_features_ : GLS_SURF_MAX_KEYPOINTS;
        std::vector<DMatch> m(static_cast<size_t>(cap));
        int32_t n = 0;
        check(gls_surf_match(s_, query_slot, train_slot, m.data(), cap, &n, stream));
        m.resize(size_t(n));
        return m;
    }

    // findMatches (SURF.hpp:65-75)
    std::vector<std::pair<Point2f, Point2f>> findMatches(int query_slot, const std::vector<KeyPoint>& keypoints1,
                                                         int train_slot, const std::vector<KeyPoint>& keypoints2,
                                                         void* stream = nullptr) {
        const std::vector<DMatch> m = matchKeyPoints(query_slot, train_slot, stream);
        std::vector<std::pair<Point2f, Point2f>> out(m.size());
        for (size_t i = 0; i < m.size(); i++) {
            const KeyPoint& a = keypoints1[size_t(m[i].query_idx)];
            const KeyPoint& b = keypoints2[size_t(m[i].train_idx)];
            out[i] = {Point2f{a.x, a.y}, Point2f{b.x, b.y}};
        }
        return out;
    }

    // the burst loop in one batch (gls_surf_register_frames)
    std::vector<std::array<float, 9>> registerFrames(const std::vector<int32_t>& ref_slots,
                                                     const std::vector<int32_t>& frame_slots, float threshold = 1,
                                                     int max_iterations = 2000, bool scale_to_full = true,
                                                     void* stream = nullptr) {
        const int nc = int(ref_slots.size()), nf = int(frame_slots.size()) / std::max(nc, 1);
        std::vector<std::array<float, 9>> H(static_cast<size_t>(nf));
        check(gls_surf_register_frames(s_, ref_slots.data(), nc, frame_slots.data(), nf, threshold, max_iterations,
                                       scale_to_full ? 1 : 0, H.empty() ? nullptr : H[0].data(), stream));
        return H;
    }

    // RawChannels (pyramidFusion.cpp:106-143) into device planes out[c]
    void rawChannels(const uint16_t* raw, int width, int height, size_t stride_bytes, BayerPattern pattern,
                     float black_level, float white_level, float exposure_multiplier, uint32_t channel_mask,
                     ImageView out[4], bool host_input = false, void* stream = nullptr) {
        check(gls_raw_channels(s_, raw, width, height, stride_bytes, int32_t(pattern), black_level, white_level,
                               exposure_multiplier, channel_mask, out, flag_if(host_input, GLS_HOST_IO), stream));
    }

    gls_surf* handle() const { return s_; }

   private:
    gls_surf* s_ = nullptr;
    int max_features_;
    int next_ = 0;
    uint32_t detect_flags_ = 0;
};

// FindHomography (Homography.hpp:26-27) on host point pairs; the detector is
// the device context. Throws std::range_error where the reference does.
inline std::array<float, 9> FindHomography(SURF& ctx, const std::vector<std::pair<Point2f, Point2f>>& matchpoints,
                                           float threshold, int max_iterations,
                                           std::vector<int>* inlier_indices = nullptr, void* stream = nullptr) {
    std::vector<float> pairs(matchpoints.size() * 4);
    for (size_t i = 0; i < matchpoints.size(); i++) {
        pairs[4 * i + 0] = matchpoints[i].first.x;
        pairs[4 * i + 1] = matchpoints[i].first.y;
        pairs[4 * i + 2] = matchpoints[i].second.x;
        pairs[4 * i + 3] = matchpoints[i].second.y;
    }
    std::array<float, 9> H{};
    std::vector<int32_t> inl(matchpoints.size());
    int32_t n = 0;
    check(gls_find_homography(ctx.handle(), pairs.data(), int32_t(matchpoints.size()), threshold, max_iterations,
                              H.data(), inl.data(), &n, stream));
    if (inlier_indices) inlier_indices->assign(inl.begin(), inl.begin() + n);
    return H;
}

// ---------------------------------------------------------------- files and bursts
// gls::image<luma_pixel_16>::read_dng_file (pipelineTest.cpp:114-115): the
// raw samples (row-major, width x height) and the metadata
inline std::vector<uint16_t> read_dng_file(const std::string& path, gls_dng_info* info) {
    check(gls_dng_read(path.c_str(), info, nullptr, 0));
    std::vector<uint16_t> raw(size_t(info->width) * size_t(info->height));
    check(gls_dng_read(path.c_str(), info, raw.data(), size_t(info->width)));
    return raw;
}

// findBursts(parseDirectory(dir)) (pyramidFusion.cpp:36-44, 166-195) over
// paths in directory order
inline std::vector<std::vector<std::string>> findBursts(const std::vector<std::string>& paths) {
    std::vector<const char*> c;
    for (const auto& p : paths) c.push_back(p.c_str());
    std::vector<int32_t> of(paths.size());
    int32_t n = 0;
    check(gls_find_bursts(c.data(), int32_t(c.size()), of.data(), &n));
    std::vector<std::vector<std::string>> bursts(size_t(n > 0 ? n : 0));
    for (size_t i = 0; i < paths.size(); i++)
        if (of[i] >= 0) bursts[size_t(of[i])].push_back(paths[i]);
    return bursts;
}

// saveFusedImage (pyramidFusion.cpp:152-164): 8-bit RGB TIFF
inline void saveFusedImage(const ImageView& fused, const std::string& path, void* stream = nullptr) {
    check(gls_write_tiff_rgb8(path.c_str(), &fused, stream));
}

// convertToGrayscale (demosaic_kernels.hpp:673-688, demosaic.metal:1707-1723)
struct convertToGrayscale {
    void operator()(const ImageView& linearImage, ImageView* grayscaleImage, const std::array<float, 3>& transform,
                    void* stream = nullptr) const {
        check(gls_convert_to_grayscale(&linearImage, transform.data(), grayscaleImage, stream));
    }
};

// ScaleHomography (Homography.hpp:29-37)
inline std::array<float, 9> ScaleHomography(const std::array<float, 9>& H, float scale) {
    std::array<float, 9> out{};
    check(gls_scale_homography(H.data(), scale, out.data()));
    return out;
}

// RegisterAndFuseKernel (demosaic_kernels.hpp:690-710)
struct RegisterAndFuseKernel {
    void operator()(const ImageView& inputImage0, const ImageView& inputImage1, ImageView* outputImage,
                    const std::array<float, 9>& homography, int count, void* stream = nullptr) const {
        check(gls_register_and_fuse(&inputImage0, &inputImage1, outputImage, homography.data(), count, stream));
    }
};

}  // namespace gls

#endif /* GLSCAM_HPP */
