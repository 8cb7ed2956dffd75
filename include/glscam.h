/*
 * glscam.h — C ABI of the B200 raw-image path (demosaic, pyramid PCA
 * block-matching denoise and reconstruct, SURF registration, burst fusion).
 *
 * Every entry point is a plain C function over plain pointers and sizes; no
 * C++ or torch type crosses this boundary and no exception escapes it.
 * Errors come back as gls_status codes, with a thread-local message from
 * gls_last_error_message().
 *
 * The functions replace the reference's C++ entry points (paths are relative
 * to the GlassCameraPublic tree):
 *   RawConverter ctor / demosaic    MetalPipeline/raw_converter.hpp:128-183,
 *                                   MetalPipeline/raw_converter.cpp:148-248
 *   PyramidProcessor<levels>        MetalPipeline/pyramid_processor.hpp:23-62,
 *                                   MetalPipeline/pyramid_processor.cpp:96-172
 *   CameraCalibration<levels>       MetalPipeline/CameraCalibration.hpp:24-39
 *   parameter structs               MetalPipeline/demosaic.hpp:28-124
 *   SURF / FindHomography           ImageRegistration/SURF.hpp:45-80,
 *                                   ImageRegistration/Homography.hpp:26-37
 *   registerAndFuse                 MetalPipeline/demosaic_kernels.hpp:690-710
 *
 * Threading: a converter is not thread-safe (the reference's RawConverter is
 * not reentrant either: one Metal queue per converter). Distinct converters
 * are independent. All device work is ordered on the stream passed in.
 */
#ifndef GLSCAM_H
#define GLSCAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace the reference's exceptions and asserts:
 *      gls_mtl.hpp:74, iPhone14WideCalibration.cpp:61,
 *      LeastSquaresHomography.cpp:382-384, demosaic_kernels.hpp:160-163) ---- */
typedef enum gls_status {
    GLS_OK = 0,
    GLS_ERR_INVALID_ARG = 1,
    GLS_ERR_OOM = 2,
    GLS_ERR_CUDA = 3,
    GLS_ERR_TIMEOUT = 4,
    GLS_ERR_DEGENERATE = 5,
    GLS_ERR_UNSUPPORTED = 6,
    GLS_ERR_RANGE = 7
} gls_status;

/* BayerPattern, demosaic.hpp:24 */
enum { GLS_GRBG = 0, GLS_GBRG = 1, GLS_RGGB = 2, GLS_BGGR = 3 };

#define GLS_MAX_LEVELS 5

/* DenoiseParameters, demosaic.hpp:33-40 */
typedef struct gls_denoise_params {
    float luma;
    float chroma;
    float chroma_boost;
    float gradient_boost;
    float gradient_threshold;
    float sharpening;
} gls_denoise_params;

/* YCbCrNLF = pair<Vector<3>, Vector<3>>, demosaic.hpp:53 (variance = a + b*Y) */
typedef struct gls_ycbcr_nlf {
    float a[3];
    float b[3];
} gls_ycbcr_nlf;

/* RawNLF = pair<Vector<4>, Vector<4>>, demosaic.hpp:51 (channels R, G, B, G2) */
typedef struct gls_raw_nlf {
    float a[4];
    float b[4];
} gls_raw_nlf;

/* RGBConversionParameters, demosaic.hpp:43-50 (GLS_POSTPROCESS) */
typedef struct gls_rgb_conversion_params {
    float contrast;                  /* 1.05 */
    float saturation;                /* 1.0 */
    float tone_curve_slope;          /* 3.5 */
    float exposure_bias;             /* EV; log2(exposure_multiplier) is added per call */
    float blacks;                    /* 0 */
    int32_t local_tone_mapping;      /* the three-band LTM mask */
} gls_rgb_conversion_params;

/* LTMParameters, demosaic.hpp:95-100 (GLS_POSTPROCESS with local tone
 * mapping). The mask takes its shadows / highlights exponents from the
 * image histogram (demosaic.metal:1510), so those two fields are carried
 * but not read, as in the reference. */
typedef struct gls_ltm_params {
    float eps;                       /* guided-filter regulariser, 0.01 */
    float shadows;
    float highlights;
    float detail[3];                 /* low, medium, high frequency band */
} gls_ltm_params;

/* DemosaicParameters, demosaic.hpp:102-124, flattened to plain data. */
typedef struct gls_demosaic_params {
    int32_t bayer_pattern;           /* GLS_GRBG .. GLS_BGGR */
    float black_level;               /* DN */
    float white_level;               /* DN */
    float exposure_multiplier;
    float lens_shading_correction;   /* 0 disables */
    float scale_mul[4];              /* per Bayer channel R, G, B, G2 */
    float rgb_cam[9];                /* row-major 3x3 */
    float xyz_rgb[9];                /* row-major 3x3, xyz_sRGB by default */
    int32_t high_noise_image;        /* RAWDenoiseParameters::highNoiseImage */
    float raw_denoise_strength;      /* RAWDenoiseParameters::strength */
    gls_raw_nlf raw_nlf;
    gls_ycbcr_nlf pyramid_nlf[GLS_MAX_LEVELS];
    gls_denoise_params denoise[GLS_MAX_LEVELS];
    int32_t levels;                  /* pyramid levels, 1..5 (the reference fixes 5) */
    int32_t iso;
    gls_rgb_conversion_params rgb_conversion;  /* GLS_POSTPROCESS only */
    gls_ltm_params ltm;                        /* GLS_POSTPROCESS with local tone mapping */
} gls_demosaic_params;

/* element types of an image view */
enum { GLS_F32 = 0, GLS_F16 = 1, GLS_U16 = 2 };

/* An image in memory: interleaved channels, row stride in bytes. */
typedef struct gls_image_view {
    void* data;
    int32_t width;
    int32_t height;
    int32_t channels;
    int32_t dtype;                   /* GLS_F32 / GLS_F16 / GLS_U16 */
    size_t stride_bytes;
} gls_image_view;

/* flags for gls_demosaic / gls_demosaic_batch / gls_pyramid_denoise */
enum {
    GLS_DENOISE = 1u << 0,       /* run the pyramid denoise (RawConverter::demosaic noiseReduction) */
    GLS_POSTPROCESS = 1u << 1,   /* display post-processing (histogram, local tone mapping, convertTosRGB) */
    GLS_FP16_STORAGE = 1u << 2,  /* FP16 planes + fused kernels + device PCA (the batched path) */
    GLS_HOST_IO = 1u << 3,       /* raw input and caller output buffers are host memory */
    GLS_SYNC = 1u << 4,          /* block until the stream has finished (the reference is synchronous) */
    GLS_HOST_PCA = 1u << 5,      /* per-level PCA eigen-solve on the host, as the reference does */
    GLS_GRAPH = 1u << 6,         /* gls_demosaic_batch: record the batch as one CUDA graph and replay it while
                                    the batch (pointers, sizes, strides, parameter bytes) stays the same */
    GLS_SURF_CORRECTED = 1u << 7, /* gls_surf_detect_and_compute: the corrected detector (see there) */
    GLS_PERSISTENT = 1u << 8,    /* gls_demosaic_batch: every pyramid level of every frame in one persistent
                                    launch (see there) */
    GLS_BM_TENSOR = 1u << 9      /* FP16 storage, stream-launched: block matching with the patch distances
                                    and the weighted sums on the tensor cores and the weights in half
                                    precision; without it the FP16 matcher computes every weight in packed
                                    FP32 (the persistent batch always does) */
};

/* Planes a converter exposes after gls_demosaic, for stage checks. */
enum {
    GLS_PLANE_SCALED_RAW = 0,    /* 1 ch, after scaleRawData (and the high-noise raw branch) */
    GLS_PLANE_GRADIENT = 1,      /* 2 ch, sampledConvolutionSobel output */
    GLS_PLANE_DEMOSAIC = 2,      /* 4 ch camera RGB after blendHighlights */
    GLS_PLANE_DESPECKLED = 3,    /* 4 ch YCbCr input of the pyramid (after despeckle) */
    GLS_PLANE_OUTPUT = 4,        /* 4 ch final camera RGB */
    GLS_PLANE_ADJ_DESPECKLED = 5, /* 3 ch FP32: dL/d(despeckled YCbCr) of the last gls_demosaic_denoise_vjp */
    GLS_PLANE_NLF_MEAN = 6,      /* 4 ch FP32, half size: 9x9 raw channel means of the last raw noise measurement */
    GLS_PLANE_NLF_VAR = 7,       /* 4 ch FP32, half size: the matching variances */
    GLS_PLANE_DENOISED_L0 = 8,   /* + level: 4 ch denoised YCbCr of a pyramid level */
    GLS_PLANE_NLF_STATS = 13     /* 4 ch FP32: 5x5 mean Y, var Y, Cb, Cr of the last YCbCr noise measurement */
};

typedef struct gls_converter gls_converter;

/* Message of the last error on this thread ("" if none). */
const char* gls_last_error_message(void);

/* Library build string (kernels, architecture). */
const char* gls_version(void);

/* Device memory the library holds (no reference counterpart; the reference
 * allocates Metal buffers per RawConverter, raw_converter.cpp:20-45): the
 * bytes of every converter, pyramid, detector and scratch buffer of this
 * process, summed over devices, and the largest such sum since the last
 * reset. reset_peak != 0 sets the peak to the current value afterwards.
 * Buffers grow to the largest frame seen and are kept until destroy. */
gls_status gls_device_memory(uint64_t* current_bytes, uint64_t* peak_bytes, int32_t reset_peak);

/* Failure detection of the persistent batch kernel (GLS_PERSISTENT; no
 * reference counterpart): runs the kernel on `device` with one eigen-solve
 * task whose covariance input no task produces, so its bounded wait runs
 * out after limit_ns. Returns GLS_ERR_TIMEOUT with the kernel's error word
 * (1 + the task type, 3 for the eigen-solve) in *err_word, the device still
 * usable; GLS_OK would mean the wait did not run out. */
gls_status gls_persistent_selftest(int32_t device, int64_t limit_ns, int32_t* err_word);

/* RawConverter(device, icc, calibrateFromImage), raw_converter.hpp:128-156.
 * icc may be NULL (xyz_sRGB). With calibrate_from_image the converter
 * measures the noise model of every frame it converts, as the reference
 * does (raw_converter.cpp:160, 188-189; pyramid_processor.cpp:113-117):
 * the raw model on the scaled frame replaces params->raw_nlf for that frame
 * (and the high-noise raw branch is off), and each pyramid level's model,
 * measured on the level before the denoise, replaces params->pyramid_nlf
 * (despeckling keeps the given level-0 model). The caller's parameters are
 * not written; gls_converter_noise_model returns the measured models. Each
 * measurement reads its result back to the host (the reference's regression
 * runs on the host), so calibrating calls are synchronous and cannot be
 * recorded with GLS_GRAPH. */
gls_status gls_converter_create(int32_t device, const uint8_t* icc, size_t icc_len,
                                int32_t calibrate_from_image, gls_converter** out);
gls_status gls_converter_destroy(gls_converter* conv);

/* RawConverter::demosaic(raw, params, noiseReduction, postProcess),
 * raw_converter.cpp:148-248. raw is width x height uint16 (stride in bytes).
 * If out->data is NULL, *out is filled with a view of the converter-owned
 * device output (4 ch RGBA, w = 0), valid until the next call on this
 * converter, as in the reference (RawProcessor.mm:75-78). Otherwise the
 * result is written to out->data in out->dtype (GLS_F32 or GLS_F16),
 * 4 channels. stream is a cudaStream_t (NULL = legacy default stream). */
gls_status gls_demosaic(gls_converter* conv, const uint16_t* raw, int32_t width, int32_t height,
                        size_t raw_stride_bytes, const gls_demosaic_params* params, uint32_t flags,
                        gls_image_view* out, void* stream);

/* One frame of a batch. */
typedef struct gls_frame_desc {
    const uint16_t* raw;
    int32_t width;
    int32_t height;
    size_t raw_stride_bytes;
    const gls_demosaic_params* params;
    gls_image_view out;
} gls_frame_desc;

/* Batched RawConverter::demosaic over frames of uneven sizes (no reference
 * counterpart: the reference converts one frame per call). Frames are
 * spread over the converter's slot streams, largest first onto the
 * least-loaded slot; slot k runs one stream priority below slot k - 1, so
 * frames finish in turn. With GLS_HOST_IO (pinned host memory for full
 * speed) each slot uploads and downloads on copy streams of its own, which
 * overlap the other frames' kernels; the call returns when the outputs are
 * in host memory. With GLS_GRAPH (caller-owned outputs, device PCA, a
 * non-default stream, at least 2 frames) the first call runs the batch and
 * records its launch sequence, copies included, as a CUDA graph; later
 * calls with the same frames, buffers and parameter values replay that
 * graph in one launch.
 * With GLS_PERSISTENT (FP16 storage, noise reduction, device buffers,
 * caller-owned outputs, device PCA, no post-processing, not a calibrating
 * converter) the frames' front ends and pyramid images run on the slot
 * streams into a pyramid per frame, then ONE launch of a persistent
 * kernel runs every level of every frame (reconstruct, covariance,
 * eigen-solve and block matching, PyramidProcessor::denoise,
 * pyramid_processor.cpp:96-172) from a device work list whose tasks wait
 * on per-level counters, then the output transforms run; it runs the
 * stream kernels' device code (the default packed-FP32 block matcher), so
 * the results are bit-identical to the stream-launched batch. The call
 * returns after the
 * kernel, with GLS_ERR_TIMEOUT if a task's wait for its inputs ran past
 * its limit (2 s). Combined with GLS_GRAPH the whole sequence is recorded
 * and replayed. */
gls_status gls_demosaic_batch(gls_converter* conv, gls_frame_desc* frames, int32_t n_frames,
                              uint32_t flags, void* stream);

/* PyramidProcessor<levels>::denoise, pyramid_processor.cpp:96-172, on a
 * YCbCr image (4 ch) and its gradient (2 ch), both device memory (or host
 * with GLS_HOST_IO). Result: 4 ch denoised YCbCr (w = kernel norm). */
gls_status gls_pyramid_denoise(gls_converter* conv, const gls_image_view* ycc,
                               const gls_image_view* gradient, const gls_demosaic_params* params,
                               uint32_t flags, gls_image_view* out, void* stream);

/* View of an internal plane of the last call (device memory). */
gls_status gls_converter_plane(gls_converter* conv, int32_t which, gls_image_view* view);

/* RawConverter::MeasureRawNLF, raw_converter.cpp:339-490: the raw noise
 * model var = a + b * value of the four Bayer channels (R, G, B, G2),
 * measured on a scaled raw frame (1 ch, GLS_F32 or GLS_F16, device memory,
 * the output of scaleRawData): basicRawNoiseStatistics' 9x9 statistics
 * (demosaic.metal:1110-1136), then the reference's two least-squares fits,
 * with a and b multiplied by exposure_multiplier^2. Synchronous. The
 * statistics stay readable as GLS_PLANE_NLF_MEAN / GLS_PLANE_NLF_VAR. */
gls_status gls_measure_raw_nlf(gls_converter* conv, const gls_image_view* scaled_raw, int32_t bayer_pattern,
                               float exposure_multiplier, gls_raw_nlf* out, void* stream);

/* PyramidProcessor::MeasureYCbCrNLF, pyramid_processor.cpp:173-324: the
 * noise model var = a + b * Y of Y, Cb and Cr measured on one YCbCr image
 * (4 ch, GLS_F32 or GLS_F16, device memory): basicNoiseStatistics' 5x5
 * statistics (demosaic.metal:1138-1159), then the two fits, scaled by
 * exposure_multiplier^2. Synchronous. The statistics stay readable as
 * GLS_PLANE_NLF_STATS. */
gls_status gls_measure_ycbcr_nlf(gls_converter* conv, const gls_image_view* ycc, float exposure_multiplier,
                                 gls_ycbcr_nlf* out, void* stream);

/* The noise models the last calibrating call measured (a converter created
 * with calibrate_from_image): the raw model and *n_levels pyramid models
 * (at most max_levels are written). dumpNoiseModel's data
 * (demosaic.hpp:70-84). */
gls_status gls_converter_noise_model(gls_converter* conv, gls_raw_nlf* raw, gls_ycbcr_nlf* pyramid,
                                     int32_t max_levels, int32_t* n_levels);

/* Strided copy between two views of equal width, height, channels and
 * dtype (no reference counterpart: the reference maps shared-storage
 * textures, gls_mtl_image.hpp:117-208). direction: GLS_COPY_D2H,
 * GLS_COPY_D2D or GLS_COPY_H2D. Synchronous for D2H. */
enum { GLS_COPY_D2H = 0, GLS_COPY_D2D = 1, GLS_COPY_H2D = 2 };
gls_status gls_copy_view(const gls_image_view* src, gls_image_view* dst, int32_t direction, void* stream);

/* PCA basis of a pyramid level from the last denoise: 25 x 8 floats,
 * row-major (pcaSpace[row][component], pyramid_processor.hpp:46). */
gls_status gls_converter_pca_basis(gls_converter* conv, int32_t level, float* basis25x8);

/* PCA patch basis (25 x 8 floats, row-major, written to basis25x8 in device
 * memory) of one 4-channel image in device memory (luma in channel 0),
 * computed without allocating device memory. No counterpart in the
 * reference: it is gls_converter_pca_basis's computation for callers that
 * cannot call cudaMalloc (a real-time capture thread that must not block in
 * the allocator; an application whose device memory is all owned by
 * another allocator). Its scratch is a fixed 11.5 MB array that every GPU
 * loading this library holds until exit, so an image may have at most
 * 262,144 patches of the 8-pixel grid (about 16.7 megapixels); larger
 * images are rejected with GLS_ERR_INVALID_ARG. Runs on the calling
 * thread's current device, asynchronously on `stream`. The first call on
 * each device looks up the scratch array's device address; make that first
 * call before any stream capture. All calls share the one array: calls
 * whose GPU work overlaps (different streams, or different host threads)
 * race on it and must be serialised by the caller. The eigen-solve runs a
 * fixed number of steps and always writes a basis; it has no status word
 * here (a non-finite eigenvector, which no finite covariance produces, is
 * not reported). */
gls_status gls_pca_basis_noalloc(const gls_image_view* image, float* basis25x8, void* stream);

/* ---- launch accounting (no reference counterpart; the reference prints
 *      wall-clock timers, pipelineTest.cpp:161-169) ----
 * Every kernel launch of a converter is counted per kernel class. With
 * profiling enabled, each launch is also bracketed by CUDA events on its
 * stream; gls_converter_stats synchronises the device and reports the
 * summed device time per class. */
typedef struct gls_kernel_stat {
    const char* name;
    uint64_t launches;
    double ms;              /* summed event time (0 unless profiling) */
} gls_kernel_stat;
gls_status gls_converter_set_profiling(gls_converter* conv, int32_t enable);
gls_status gls_converter_stats(gls_converter* conv, gls_kernel_stat* stats, int32_t max_stats, int32_t* n_stats);
gls_status gls_converter_reset_stats(gls_converter* conv);

/* The grain tables of the display post-processing (Noise2D::randomSeed +
 * initGradients, SimplexNoise.hpp:109-143): perm[514] and grad[514][2] for
 * a seed (the raw frame's first pixel). The same code builds them on the
 * device during gls_demosaic with GLS_POSTPROCESS. */
gls_status gls_grain_tables(uint32_t seed, int32_t* perm, float* grad);

/* Decisions of the FP16 block matcher's tile autotuner (no reference
 * counterpart): for each pyramid level size met so far in this process,
 * (width, height, variant), variant = 10 x thread rows + pixels per thread:
 * 84 and 162 for 32x32-pixel tiles, 44 and 82 for 32x16. The first frame of
 * a size times every variant and keeps the fastest; all compute identical
 * results. Writes at most max_entries triples to entries; *n receives the
 * count. GLS_BM_TILE=84, 44, 82 or 162 in the environment (8 or 4 for 84 or
 * 44) fixes the variant. */
gls_status gls_block_match_tiles(int32_t* entries, int32_t max_entries, int32_t* n);

/* ---- CameraCalibration<levels> (CameraCalibration.hpp:24-39) ----
 * Fills the noise model and the denoise schedule of a built-in camera for
 * an ISO, as nlfFromIso() + getDenoiseParameters() do. Returns GLS_ERR_RANGE
 * for an ISO the calibration does not cover. */
enum { GLS_CAMERA_IPHONE14_WIDE = 0 };
gls_status gls_calibration_fill(int32_t camera, int32_t iso, gls_demosaic_params* params);

/* ==== DNG ingest (no live reference code: the reference reads DNGs with
 * the un-vendored GlassImage library, gls::image::read_dng_file, used at
 * pipelineTest.cpp:114-115 and pyramidFusion.cpp:50, 297, 322) ====
 * A self-contained TIFF/DNG reader for the CFA raw image of a DNG: the raw
 * IFD is the first IFD (IFD0 or a SubIFD) with NewSubFileType 0 and CFA
 * photometric interpretation; its samples are uncompressed (8, 16 or
 * 10/12/14-bit packed MSB first, rows byte-aligned) or lossless JPEG
 * (ITU-T T.81 process 14, predictors 1-7, any component interleave; DNG
 * Compression 7), in strips or tiles; tiles are decoded in parallel on the
 * host. gls_dng_info carries the metadata unpackDNGMetadata and
 * CameraCalibration::getDemosaicParameters read (demosaic_utils.cpp:268-366,
 * CameraCalibration.cpp:25-58). */
typedef struct gls_dng_info {
    int32_t width, height;              /* raw image */
    int32_t bits_per_sample;
    int32_t compression;                /* 1 or 7 */
    uint8_t cfa_pattern[4];             /* CFAPattern (0 R, 1 G, 2 B) */
    int32_t bayer_pattern;              /* GLS_GRBG .. GLS_BGGR, from cfa_pattern as the reference maps it */
    float black_level;                  /* BlackLevel[0], 0 if absent */
    float white_level;                  /* WhiteLevel[0], 65535 if absent */
    float baseline_exposure;            /* BaselineExposure (EV), 0 if absent */
    int32_t has_color_matrix1, has_color_matrix2, has_as_shot_neutral;
    float color_matrix1[9], color_matrix2[9]; /* XYZ -> camera, row-major */
    float as_shot_neutral[3];
    int32_t calibration_illuminant1, calibration_illuminant2;
    int32_t iso;                        /* EXIF RecommendedExposureIndex, else ISOSpeedRatings, else 0 */
    float exposure_time;                /* EXIF ExposureTime (s), 0 if absent */
    int32_t active_area[4];             /* top, left, bottom, right (the whole image if absent) */
    char make[64], model[64], lens_model[96];
} gls_dng_info;

/* Reads a DNG's raw image and metadata. With raw NULL only *info is filled
 * (to size the buffer). raw: width x height uint16 host memory, row stride
 * raw_stride_elems (>= width). */
gls_status gls_dng_read(const char* path, gls_dng_info* info, uint16_t* raw, size_t raw_stride_elems);

/* Writes raw (width x height uint16, host) as a DNG carrying info's
 * metadata (a single CFA IFD0 with an EXIF IFD): compression 1
 * (uncompressed 16-bit) or 7 (lossless JPEG, predictor 1, tiles of
 * tile_size x tile_size, two components per row as DNG writers interleave
 * Bayer rows; tile_size 0: one strip). The reference captures DNGs through
 * the operating system; this writer exists for round trips and tests. */
gls_status gls_dng_write(const char* path, const gls_dng_info* info, const uint16_t* raw, size_t raw_stride_elems,
                         int32_t compression, int32_t tile_size);

/* CameraCalibration::getDemosaicParameters (CameraCalibration.cpp:25-58)
 * with unpackDNGMetadata (demosaic_utils.cpp:268-366) without automatic
 * white balance: black and white levels, Bayer pattern, exposure
 * multiplier (2^BaselineExposure, at most 1; scale_mul takes the rest),
 * rgb_cam from ColorMatrix2 (else ColorMatrix1) and xyz_rgb
 * (cam_xyz_coeff, demosaic_utils.cpp:78-101), the white balance from
 * AsShotNeutral (else the matrix's white), scale_mul, then the camera's
 * noise model and denoise schedule at the EXIF ISO. camera: a
 * GLS_CAMERA_* id. xyz_rgb may be NULL (sRGB). Returns GLS_ERR_RANGE for a
 * singular colour matrix or an ISO the calibration does not cover. */
gls_status gls_dng_demosaic_params(const gls_dng_info* info, const float* xyz_rgb, int32_t camera,
                                   gls_demosaic_params* params);

/* The camera a DNG was taken with, as pipelineTest.cpp:133-160 selects it
 * (Apple iPhone 14 Pro / Pro Max by lens model; unknown lenses use the
 * wide camera): a GLS_CAMERA_* id, or -1 for a device without a
 * calibration. */
int32_t gls_dng_camera(const gls_dng_info* info);

/* ==== Burst driver host side (PyramidFusion/pyramidFusion.cpp) ==== */

/* findBursts (pyramidFusion.cpp:166-195) over paths in directory order
 * (parseDirectory sorts them, :36-44): a file whose stem contains "_1_"
 * starts a burst; later files join it when their stem has the same prefix
 * up to that position. burst_of[i] receives file i's burst (0, 1, ...) or
 * -1; *n_bursts the number of bursts. */
gls_status gls_find_bursts(const char* const* paths, int32_t n, int32_t* burst_of, int32_t* n_bursts);

/* convertToGrayscale (demosaic.metal:1707-1723), the luma image
 * PyramidFusion's main_full registers on (convertImage,
 * pyramidFusion.cpp:80-98, transform = rgb_cam's first row):
 * gray = max(t . ((rgb - 0.1) / 0.9), 0). rgb: 4 ch F32/F16, gray: 1 ch
 * F32, both device memory; asynchronous on stream. */
gls_status gls_convert_to_grayscale(const gls_image_view* rgb, const float* transform, gls_image_view* gray,
                                    void* stream);

/* saveFusedImage (pyramidFusion.cpp:152-164): an RGBA (or RGB) F32/F16
 * image, host or device memory, written as an uncompressed 8-bit RGB TIFF
 * with (uint8) (255 * clamp(v, 0, 1)) per channel. */
gls_status gls_write_tiff_rgb8(const char* path, const gls_image_view* rgba, void* stream);

/* Gaussian kernel folded into bilinear taps (weight, dx, dy) per tap,
 * gaussianKernelBilinearWeights, demosaic_utils.cpp:987-1006. Writes at
 * most max_taps taps; *n_taps receives the count. */
gls_status gls_gaussian_bilinear_taps(float radius, float* taps, int32_t max_taps, int32_t* n_taps);

/* ==== Adjoint (no reference counterpart) ====
 * Gradient of L = mean over pixels and R, G, B of (output - target)^2, where
 * output is the FP32 path's linear camera RGB of `raw` (demosaic + pyramid
 * denoise + reconstruct), with respect to GLS_ADJ_NPARAMS scalars of
 * gls_demosaic_params, laid out as:
 *   [GLS_ADJ_LUMA + l]     denoise[l].luma
 *   [GLS_ADJ_CHROMA + l]   denoise[l].chroma
 *   [GLS_ADJ_NLF_AY + l]   pyramid_nlf[l].a[0]
 *   [GLS_ADJ_NLF_BY + l]   pyramid_nlf[l].b[0]
 *   [GLS_ADJ_NLF_AC + l]   pyramid_nlf[l].a[1] = a[2] (Cb and Cr tied)
 *   [GLS_ADJ_NLF_BC + l]   pyramid_nlf[l].b[1] = b[2]
 *   [GLS_ADJ_RAW_GREEN_A]  raw_nlf.a[1] and a[3] moved together (their mean,
 *                          the demosaic's green variance offset)
 *   [GLS_ADJ_RAW_GREEN_B]  raw_nlf.b[1] and b[3] moved together (the green
 *                          variance slope of the demosaic and of the
 *                          high-noise cross denoise)
 * for l < levels (entries of absent levels are 0). The forward runs first
 * (as gls_demosaic with GLS_DENOISE on FP32 planes); the reverse sweep of
 * the pyramid is hand-written CUDA over its retained planes, with each
 * level's PCA basis held fixed, down to dL/d(despeckled image)
 * (GLS_PLANE_ADJ_DESPECKLED afterwards); the raw front end (cross denoise,
 * demosaic, despeckle) contributes by forward-mode tangents along the two
 * raw-green parameters. The gradient plane's dependence on them (a blur
 * radius switch) is piecewise constant and contributes nothing.
 * target: GLS_F32 RGB or RGBA, width x height, device memory (host with
 * GLS_HOST_IO, which also makes raw host memory). Synchronises the stream. */
#define GLS_ADJ_NPARAMS 32
enum {
    GLS_ADJ_LUMA = 0,
    GLS_ADJ_CHROMA = 5,
    GLS_ADJ_NLF_AY = 10,
    GLS_ADJ_NLF_BY = 15,
    GLS_ADJ_NLF_AC = 20,
    GLS_ADJ_NLF_BC = 25,
    GLS_ADJ_RAW_GREEN_A = 30,
    GLS_ADJ_RAW_GREEN_B = 31
};
gls_status gls_demosaic_denoise_vjp(gls_converter* conv, const uint16_t* raw, int32_t width, int32_t height,
                                    size_t raw_stride_bytes, const gls_demosaic_params* params,
                                    const gls_image_view* target, uint32_t flags, double* loss, float* grad,
                                    void* stream);

/* Vector-Jacobian product of PyramidProcessor<levels>::denoise (no
 * reference counterpart; the denoise-only counterpart of
 * gls_demosaic_denoise_vjp, as gls_pyramid_denoise is of gls_demosaic).
 * The FP32 denoise of ycc (4 ch YCbCr) and gradient (2 ch) runs first, as
 * gls_pyramid_denoise without GLS_FP16_STORAGE. Given g_out = dL/d(denoised
 * Y, Cb, Cr) (GLS_F32, 3 or 4 channels, a fourth ignored), grad receives
 * GLS_ADJ_NPARAMS entries, dL/dtheta of the pyramid parameters (the
 * raw-green entries are 0: they act before this stage), and g_ycc, unless
 * NULL, dL/d(ycc) (GLS_F32, 3 or 4 channels; a fourth is written 0). Each
 * level's PCA basis is held fixed. Views are device memory, or host memory
 * with GLS_HOST_IO. Synchronises the stream. */
gls_status gls_pyramid_denoise_vjp(gls_converter* conv, const gls_image_view* ycc, const gls_image_view* gradient,
                                   const gls_demosaic_params* params, const gls_image_view* g_out, uint32_t flags,
                                   float* grad, gls_image_view* g_ycc, void* stream);

/* ==== Registration and fusion (ImageRegistration/, PyramidFusion/) ==== */

/* KeyPoint (ImageRegistration/feature2d.hpp:25-47), 28 bytes. angle is in
 * radians, as the reference stores it; size == -1 marks a keypoint whose
 * orientation could not be sampled (SURF.cpp:529-554). */
typedef struct gls_keypoint {
    float x, y, size, angle, response;
    int32_t octave, class_id;
} gls_keypoint;

/* DMatch (ImageRegistration/SURF.hpp:29-42) */
typedef struct gls_match {
    int32_t query_idx, train_idx;
    float distance;
} gls_match;

typedef struct gls_surf gls_surf;

/* Feature slots a detector holds (detectAndCompute results kept on the
 * device for matching). */
#define GLS_SURF_SLOTS 32
/* Most keypoints one detection keeps before the max_features cut
 * (KeyPointMaxima::MaxCount, SURF.cpp:870-874). */
#define GLS_SURF_MAX_KEYPOINTS 64000

/* SURF::makeInstance (SURF.hpp:45-47, SURF.cpp:1082-1112): a detector for
 * width x height single-channel F32 images on a CUDA device. max_features
 * < 0 keeps every keypoint. The reference's defaults are 4 octaves, 2
 * layers per octave, threshold 0.02. */
gls_status gls_surf_create(int32_t device, int32_t width, int32_t height, int32_t max_features, int32_t n_octaves,
                           int32_t n_octave_layers, float hessian_threshold, gls_surf** out);
gls_status gls_surf_destroy(gls_surf* s);

/* SURF::detectAndCompute (SURF.hpp:57-58, SURF.cpp:1380-1450, one
 * section): integral image, fast-Hessian detector, KeypointGreater order,
 * max_features cut, orientation and 64-D descriptor, into feature slot
 * `slot`. img: F32, 1 channel, width x height, device memory or host
 * memory with GLS_HOST_IO. Asynchronous on `stream` unless GLS_SYNC or
 * GLS_HOST_IO.
 * By default the reference's detector, two defects included: the maxima
 * interpolation adds the scale offset to x, y and size alike (SURF.metal:200
 * returns `(float3)(a, b, c) / det`, a C++ comma expression), and of K > 32
 * keypoints only the first min(K, ceil(K/8)^2) are oriented and described
 * (SURF.cpp:681-693; the others keep angle -1 and a zero descriptor).
 * GLS_SURF_CORRECTED solves the interpolation per axis and describes every
 * keypoint. */
gls_status gls_surf_detect_and_compute(gls_surf* s, const gls_image_view* img, int32_t slot, uint32_t flags,
                                       void* stream);

/* Copies a slot's keypoints, and its descriptors ([n][64] floats) when desc
 * is not NULL, to host memory; synchronises the stream. *n receives the
 * keypoint count; at most `capacity` are written. */
gls_status gls_surf_features(gls_surf* s, int32_t slot, gls_keypoint* kps, float* desc, int32_t capacity, int32_t* n,
                             void* stream);

/* Loads n keypoints and their descriptors ([n][64] floats), as
 * gls_surf_features returns them, into a feature slot, for matching
 * against features another detector (another GPU) computed: a burst split
 * over ranks receives the reference frame's features by broadcast instead
 * of detecting them again. Device pointers, or host pointers with
 * GLS_HOST_IO (then synchronous). n <= the detector's max_features. */
gls_status gls_surf_load_features(gls_surf* s, int32_t slot, const gls_keypoint* kps, const float* desc, int32_t n,
                                  uint32_t flags, void* stream);

/* Device view of a detector plane: GLS_SURF_PLANE_INTEGRAL is the summed-area
 * table of the last detection, (width+1) x (height+1) F32 with a zero first
 * row and column (integralImageKernel, SURF.cpp:776-825). */
enum { GLS_SURF_PLANE_INTEGRAL = 0 };
gls_status gls_surf_plane(gls_surf* s, int32_t which, gls_image_view* view);

/* SURF::matchKeyPoints (SURF.cpp:931-974, SURF.metal:423-487): for every
 * keypoint of query_slot its nearest descriptor in train_slot, sorted by
 * distance then query index (refineMatch). The result stays in the
 * detector for gls_surf_find_homography; with matches != NULL it is also
 * copied to host memory (synchronising) and *n receives the count. */
gls_status gls_surf_match(gls_surf* s, int32_t query_slot, int32_t train_slot, gls_match* matches, int32_t capacity,
                          int32_t* n, void* stream);

/* FindHomography (Homography.cpp:72-116) over the last match result, as
 * SURF::findMatches pairs it (query point -> train point): RANSAC with
 * max_iterations 4-point least-squares models (samples from std::mt19937
 * with its default seed, uniform integers by mask-and-reject), inliers at
 * squared error < threshold refitted by FindLeastSquaresHomography. Runs
 * on the GPU; H (row-major, 9 floats) and the inlier indices are copied to
 * host memory (synchronising). *n_inliers receives the count; inliers may
 * be NULL. */
gls_status gls_surf_find_homography(gls_surf* s, float threshold, int32_t max_iterations, float* H,
                                    int32_t* inliers, int32_t* n_inliers, void* stream);

/* The same for n host point pairs (x1, y1, x2, y2), with the detector as
 * the device context. */
gls_status gls_find_homography(gls_surf* ctx, const float* pairs, int32_t n, float threshold, int32_t max_iterations,
                               float* H, int32_t* inliers, int32_t* n_inliers, void* stream);

/* Burst registration in one batch (the per-frame loop of
 * pyramidFusion.cpp:318-346): for frame f and channel c, the features of
 * slot frame_slots[f * n_channels + c] are matched against reference slot
 * ref_slots[c] and FindHomography runs on the pairs; all n_frames x
 * n_channels (at most 64) problems go to the GPU together. The channel
 * homographies of a frame are averaged as the reference does
 * (H = (H_c + H * c) / (c + 1)) and, with scale_to_full, mapped by
 * ScaleHomography. H receives [n_frames][9] floats in host memory;
 * synchronises the stream. */
gls_status gls_surf_register_frames(gls_surf* s, const int32_t* ref_slots, int32_t n_channels,
                                    const int32_t* frame_slots, int32_t n_frames, float threshold,
                                    int32_t max_iterations, int32_t scale_to_full, float* H, void* stream);

/* ScaleHomography (Homography.hpp:29-37): S H S^-1 with S = diag(2, 2, 1);
 * like the reference, the scale argument does not enter. */
gls_status gls_scale_homography(const float* H, float scale, float* out);

/* RawChannels (PyramidFusion/pyramidFusion.cpp:106-143): the Bayer
 * channels selected by channel_mask (bit c: 0 = R, 1 = G, 2 = B, 3 = G2 by
 * the host table demosaic.hpp:128-133) at half resolution, through
 * toneCurve(clamp(exposure (v - black) / white, 0, 1), 3.5), as F32 planes
 * out[c] (device memory, (width/2) x (height/2)). raw is device memory, or
 * host memory with GLS_HOST_IO. */
gls_status gls_raw_channels(gls_surf* ctx, const uint16_t* raw, int32_t width, int32_t height, size_t stride_bytes,
                            int32_t bayer_pattern, float black_level, float white_level, float exposure_multiplier,
                            uint32_t channel_mask, gls_image_view* out, uint32_t flags, void* stream);

/* registerAndFuse (SURF.metal:489-516, RegisterAndFuseKernel
 * demosaic_kernels.hpp:690-710): out = ((count - 1) fused + input(H p)) /
 * count per pixel, input sampled bilinearly with clamp-to-edge at H (x, y).
 * fused / out: F32 RGBA (out may alias fused); input: F32 or F16 RGBA of
 * any size; H: host, row-major. */
gls_status gls_register_and_fuse(const gls_image_view* fused, const gls_image_view* input, gls_image_view* out,
                                 const float* H, int32_t count, void* stream);

/* registerImage (SURF.metal:518-538): out = input(H p). */
gls_status gls_register_image(const gls_image_view* input, gls_image_view* out, const float* H, void* stream);

/* Pyramid burst fusion (the reference declares this API but leaves it
 * unimplemented, pyramid_processor.hpp:51-55, 64-70; this is the library's
 * design). frames[0] is the reference; frame f > 0 is pull-warped into it
 * by H[f] (row-major 3x3, reference -> frame, as registerAndFuse takes;
 * H[0] is not read). Each warped frame is split into a `levels`-level
 * Laplacian pyramid with the denoiser's down- and up-sampling; per level
 * and pixel the frames are averaged with weights
 * exp(-robustness * |band - reference band|^2) (the reference weighs 1),
 * and the fused pyramid is collapsed. robustness = 0 gives uniform weights,
 * whose result is the flat mean of the warped frames (registerAndFuse's,
 * up to float rounding). frames: RGBA GLS_F32 or GLS_F16 device views;
 * out: width x height RGBA GLS_F32 or GLS_F16 device view (alpha 0). */
gls_status gls_fuse_pyramid(gls_surf* ctx, const gls_image_view* frames, int32_t n_frames, const float* H,
                            int32_t levels, float robustness, gls_image_view* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GLSCAM_H */
