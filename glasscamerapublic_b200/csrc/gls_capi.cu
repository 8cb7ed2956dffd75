// gls_capi.cu — the converter object and the extern "C" entry points of
// include/glscam.h. The host sequence follows RawConverter::demosaic
// (raw_converter.cpp:148-248) and PyramidProcessor<levels>::denoise
// (pyramid_processor.cpp:96-172); the kernels are in gls_front.cu and
// gls_pyramid.cu.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "gls_common.cuh"
#include "gls_devbuf.h"
#include "gls_host.h"
#include "gls_kernels.h"
#include "gls_noise.h"

namespace gls {

static thread_local std::string g_last_error;

gls_status set_error(gls_status code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
void clear_error() { g_last_error.clear(); }

static std::atomic<long long> g_dev_bytes{0}, g_dev_peak{0};

void devbuf_account(long long delta) {
    const long long now = g_dev_bytes.fetch_add(delta) + delta;
    long long pk = g_dev_peak.load();
    while (now > pk && !g_dev_peak.compare_exchange_weak(pk, now)) {
    }
}

cudaError_t ensure_dynamic_smem(const void* func, int bytes) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({func, dev})) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.insert({func, dev});
    return e;
}

template <class S, int C>
static Plane<S, C> plane(DevBuf& b, int w, int h) {
    return Plane<S, C>{reinterpret_cast<S*>(b.p), w, h, size_t(w) * C};
}

// Device state of one storage type: every plane of RawConverter and
// PyramidProcessor (raw_converter.hpp:84-104, pyramid_processor.hpp:42-48).
template <class S>
struct Pipeline {
    int W = 0, H = 0, L = 0;
    DevBuf raw, scaled, grad, quad, A, B, pca, acc, basis, status;
    DevBuf scaled0;  // the Bayer plane before the raw branch, kept only for the adjoint
    DevBuf post_hist, post_stats, post_perm, post_gtab, post_ab;  // display post-processing scratch
    // the pyramid: each level's image and gradient (level 0 in B / grad) and
    // denoised output; one reconstructed layer buffer serves every level
    // (a level's layer is read only by that level's PCA and block matching;
    // the adjoint recomputes it in its reverse sweep)
    DevBuf img[GLS_MAX_LEVELS], gradp[GLS_MAX_LEVELS], den[GLS_MAX_LEVELS], layer;
    DevBuf nc[GLS_MAX_LEVELS];  // chroma norms, kept only for the adjoint
    DevBuf out_f32, out_f16, stage_in, stage_grad;
    size_t acc_off[GLS_MAX_LEVELS] = {};  // per level: the first covariance partial (doubles into acc)
    std::vector<double> host_acc;
    std::vector<float> host_basis;

    gls_status ensure(int w, int h, int levels) {
        const size_t n = size_t(w) * h;
        GLS_TRY(raw.ensure(n * sizeof(uint16_t)));
        GLS_TRY(scaled.ensure(n * sizeof(S)));
        GLS_TRY(grad.ensure(n * 2 * sizeof(S)));
        GLS_TRY(quad.ensure((n / 4 + 1) * 4 * sizeof(S)));
        GLS_TRY(A.ensure(n * 4 * sizeof(S)));
        GLS_TRY(B.ensure(n * 4 * sizeof(S)));
        GLS_TRY(pca.ensure(n * 8 * sizeof(S)));
        GLS_TRY(layer.ensure(n * 4 * sizeof(S)));
        size_t rows = 0;
        for (int i = 0; i < levels; i++) {
            acc_off[i] = rows * kPcaAcc;
            rows += size_t(pca_cov_rows(w >> i, h >> i));
        }
        GLS_TRY(acc.ensure(sizeof(double) * kPcaAcc * std::max<size_t>(rows, 1)));
        GLS_TRY(basis.ensure(sizeof(float) * 200 * GLS_MAX_LEVELS));
        GLS_TRY(status.ensure(sizeof(int) * GLS_MAX_LEVELS));
        for (int i = 0; i < levels; i++) {
            const size_t ni = size_t(w >> i) * (h >> i);
            if (i > 0) {
                GLS_TRY(img[i].ensure(ni * 4 * sizeof(S)));
                GLS_TRY(gradp[i].ensure(ni * 2 * sizeof(S)));
            }
            GLS_TRY(den[i].ensure(ni * 4 * sizeof(S)));
        }
        W = w;
        H = h;
        L = levels;
        return GLS_OK;
    }
    void release() {
        for (DevBuf* b : {&raw, &scaled, &scaled0, &grad, &quad, &A, &B, &pca, &layer, &acc, &basis, &status, &out_f32,
                          &out_f16, &stage_in, &stage_grad, &post_hist, &post_stats, &post_perm, &post_gtab, &post_ab})
            b->release();
        for (int i = 0; i < GLS_MAX_LEVELS; i++) {
            img[i].release();
            gradp[i].release();
            den[i].release();
            nc[i].release();
        }
    }
};

}  // namespace gls

using namespace gls;

namespace gls {
// kernel classes for launch accounting
enum KernelClass {
    KC_SCALE, KC_SOBEL_BLUR, KC_RAW_DENOISE, KC_DEMOSAIC, KC_DESPECKLE, KC_DOWNSAMPLE, KC_SUBTRACT,
    KC_PCA_COV, KC_PCA_EIGEN, KC_PCA_PROJECT, KC_BLOCK_MATCH, KC_OUTPUT, KC_VIEW_IN, KC_POST, KC_NLF,
    KC_PERSISTENT, KC_COUNT
};
static const char* const kKcNames[KC_COUNT] = {
    "scale_raw", "sobel_blur", "raw_quad_denoise", "demosaic", "despeckle", "downsample", "subtract_noise",
    "pca_cov", "pca_eigen", "pca_project", "block_match", "output_transform", "view_in", "post_process", "noise_model",
    "pyramid_persistent"};

struct Prof {
    bool on = false;
    uint64_t launches[KC_COUNT] = {};
    double ms[KC_COUNT] = {};
    struct Pending {
        int kc;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void drain() {  // device must be synchronised
        for (auto& p : pending) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) ms[p.kc] += t;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    ~Prof() {
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// Counts the launches of one kernel class and, when profiling, brackets
// them with events on the launch stream.
struct KScope {
    Prof& pr;
    int kc;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    KScope(Prof& p, int k, cudaStream_t st, int n = 1) : pr(p), kc(k), s(st) {
        pr.launches[kc] += n;
        if (pr.on) {
            a = pr.get();
            cudaEventRecord(a, s);
        }
    }
    ~KScope() {
        if (pr.on) {
            cudaEvent_t b = pr.get();
            cudaEventRecord(b, s);
            pr.pending.push_back({kc, a, b});
        }
    }
};
}  // namespace gls

// Frames of a batch run concurrently on kSlots streams, each slot with its
// own planes (about 0.7 GB per slot at 12 MP in FP16); slot 0 also serves
// the single-frame calls. Six slots: a 6-frame 12 MP batch runs 1% faster
// than with three (more single-block kernels of one frame overlap other
// frames' work), 2.5% faster than with two.
constexpr int kSlots = 6;

struct gls_converter {
    int device = 0;
    Prof prof;
    Pipeline<float> p32s[kSlots];
    Pipeline<__half> p16s[kSlots];
    Pipeline<float>& p32 = p32s[0];
    Pipeline<__half>& p16 = p16s[0];
    cudaStream_t slot_stream[kSlots] = {};
    // host I/O of a batch: per slot, copy streams and the events that order
    // them against the slot's kernels (staging buffers released / filled)
    cudaStream_t cin_stream[kSlots] = {}, cout_stream[kSlots] = {};
    cudaEvent_t raw_free[kSlots] = {}, raw_ready[kSlots] = {}, out_ready[kSlots] = {}, out_free[kSlots] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kSlots] = {};
    int last_storage = -1;  // GLS_F32 / GLS_F16 of the last single-frame call
    int last_levels = 0;
    int last_w = 0, last_h = 0;
    bool last_denoise = false;
    bool keep_nc = false;  // the FP32 forward keeps its chroma norms (for the adjoint)
    // the last GLS_GRAPH batch: its signature and executable graph
    std::vector<uint64_t> graph_key;
    cudaGraphExec_t graph_exec = nullptr;
    bool graph_persistent = false;  // the recorded batch reads the persistent kernel's error word
    // GLS_PERSISTENT batches: a pyramid per frame, the work list of the last
    // batch (its signature, descriptors, tasks) and the kernel's counters
    std::vector<std::unique_ptr<Pipeline<__half>>> pframes;
    std::vector<uint64_t> plan_key;
    int plan_tasks = 0, plan_levels = 0, plan_grid = 0;
    DevBuf plan_task_buf, plan_level_buf, plan_cnt, plan_ctl;  // ctl: next, err
    // adjoint scratch (gls_demosaic_denoise_vjp)
    DevBuf adj_gden[2], adj_rec, adj_glayer, adj_gpca, adj_gup, adj_part, adj_loss, adj_target;
    DevBuf adj_gimg, adj_gp1, adj_jvp, adj_jvp_part;  // dL/d(input pyramid), front-end tangents
    DevBuf adj_gout;                                   // a caller's cotangent, packed (pyramid VJP)
    int adj_gimg_w = 0, adj_gimg_h = 0;                // size of the last dL/d(despeckled image)
    // noise-model measurement (calibrateFromImage): scratch, the last
    // statistics planes and the last measured models
    bool calibrate = false;
    DevBuf nlf_scratch, nlf_mean, nlf_var, nlf_stats;
    int nlf_mw = 0, nlf_mh = 0, nlf_sw = 0, nlf_sh = 0;
    gls_raw_nlf nlf_raw{};
    gls_ycbcr_nlf nlf_pyr[GLS_MAX_LEVELS]{};
    int nlf_levels = 0;
};

namespace gls {

// ---- view conversion kernels (caller views <-> internal planes)
template <class I, class S, int C>
__global__ void k_view_in(const I* __restrict__ src, size_t pitch, Plane<S, C> dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dst.w || y >= dst.h) return;
    const I* s = src + size_t(y) * pitch + size_t(x) * C;
    S* d = dst.px(x, y);
#pragma unroll
    for (int c = 0; c < C; c++) d[c] = from_f<S>(to_f(s[c]));
}

template <class S, int C>
static gls_status view_to_plane(const gls_image_view* v, bool host_io, DevBuf& stage, Plane<S, C> dst, cudaStream_t s) {
    if (v->channels != C) return set_error(GLS_ERR_INVALID_ARG, "view has %d channels, expected %d", v->channels, C);
    if (v->dtype != GLS_F32 && v->dtype != GLS_F16) return set_error(GLS_ERR_INVALID_ARG, "view dtype must be F32 or F16");
    const size_t es = v->dtype == GLS_F32 ? 4 : 2;
    const size_t row = size_t(v->width) * C * es;
    if (v->stride_bytes < row || v->stride_bytes % es) return set_error(GLS_ERR_INVALID_ARG, "bad view stride");
    const void* src = v->data;
    size_t pitch = v->stride_bytes / es;
    if (host_io) {
        GLS_TRY(stage.ensure(row * v->height));
        GLS_CUDA(cudaMemcpy2DAsync(stage.p, row, v->data, v->stride_bytes, row, v->height, cudaMemcpyHostToDevice, s));
        src = stage.p;
        pitch = size_t(v->width) * C;
    }
    dim3 b(32, 8), g((dst.w + 31) / 32, (dst.h + 7) / 8);
    if (v->dtype == GLS_F32) k_view_in<float, S, C><<<g, b, 0, s>>>(static_cast<const float*>(src), pitch, dst);
    else k_view_in<__half, S, C><<<g, b, 0, s>>>(static_cast<const __half*>(src), pitch, dst);
    GLS_CUDA(cudaGetLastError());
    return GLS_OK;
}

static gls_status check_params(const gls_demosaic_params* p, int w, int h) {
    if (!p) return set_error(GLS_ERR_INVALID_ARG, "params is NULL");
    if (p->bayer_pattern < 0 || p->bayer_pattern > 3) return set_error(GLS_ERR_INVALID_ARG, "bad bayer_pattern %d", p->bayer_pattern);
    if (p->levels < 1 || p->levels > GLS_MAX_LEVELS) return set_error(GLS_ERR_INVALID_ARG, "levels must be 1..5 (got %d)", p->levels);
    if (w < 4 || h < 4 || (w & 1) || (h & 1))
        return set_error(GLS_ERR_INVALID_ARG, "image must be at least 4x4 with even width and height (got %dx%d)", w, h);
    if ((w >> (p->levels - 1)) < 1 || (h >> (p->levels - 1)) < 1)
        return set_error(GLS_ERR_INVALID_ARG, "image %dx%d too small for %d pyramid levels", w, h, p->levels);
    if (!(p->white_level > p->black_level)) return set_error(GLS_ERR_INVALID_ARG, "white_level must exceed black_level");
    return GLS_OK;
}

// Output of the final stage: either the caller's buffer (device, or host
// through the converter's internal plane) or the converter's own plane.
template <class O>
struct OutTarget {
    Plane<O, 4> plane;
    bool copy_to_host = false;
    void* host = nullptr;
    size_t host_stride = 0;
};

// The display post-processing reads the histogram of denoised level 3 and
// guides the tone mapping with levels 4, 2 and 0: the reference's 5-level
// pyramid (raw_converter.cpp:88-110).
static gls_status check_post(const gls_demosaic_params* p, uint32_t flags) {
    if (!(flags & GLS_POSTPROCESS) || !(flags & GLS_DENOISE) || !p) return GLS_OK;
    if (p->levels != 5) return set_error(GLS_ERR_INVALID_ARG, "post-processing needs the 5-level pyramid");
    return GLS_OK;
}

// RawConverter::MeasureRawNLF / PyramidProcessor::MeasureYCbCrNLF on the
// device (gls_nlf.cu), the result read back to the host (synchronous, as the
// reference's host regressions are)
static gls_status nlf_result(gls_converter* cv, gls_raw_nlf* host, cudaStream_t s) {
    GLS_CUDA(cudaGetLastError());
    const auto* dres = reinterpret_cast<const gls_raw_nlf*>(static_cast<char*>(cv->nlf_scratch.p) + nlf_scratch_bytes());
    GLS_CUDA(cudaMemcpyAsync(host, dres, sizeof(gls_raw_nlf), cudaMemcpyDeviceToHost, s));
    GLS_CUDA(cudaStreamSynchronize(s));
    return GLS_OK;
}

template <class S>
static gls_status measure_raw_nlf(gls_converter* cv, Plane<S, 1> scaled, int pattern, float exposure,
                                  gls_raw_nlf* out, cudaStream_t s) {
    const int mw = scaled.w / 2, mh = scaled.h / 2;
    if (mw < 1 || mh < 1) return set_error(GLS_ERR_INVALID_ARG, "raw noise measurement needs a frame of at least 2 x 2");
    GLS_TRY(cv->nlf_scratch.ensure_zeroed(nlf_scratch_bytes() + sizeof(gls_raw_nlf), s));
    GLS_TRY(cv->nlf_mean.ensure(size_t(mw) * mh * 4 * sizeof(float)));
    GLS_TRY(cv->nlf_var.ensure(size_t(mw) * mh * 4 * sizeof(float)));
    auto* dres = reinterpret_cast<gls_raw_nlf*>(static_cast<char*>(cv->nlf_scratch.p) + nlf_scratch_bytes());
    {
        KScope k(cv->prof, KC_NLF, s, 0);
        cv->prof.launches[KC_NLF] += launch_measure_raw_nlf<S>(scaled, pattern, plane<float, 4>(cv->nlf_mean, mw, mh),
                                                               plane<float, 4>(cv->nlf_var, mw, mh), exposure,
                                                               cv->nlf_scratch.p, dres, s);
    }
    cv->nlf_mw = mw;
    cv->nlf_mh = mh;
    return nlf_result(cv, out, s);
}

template <class S>
static gls_status measure_ycc_nlf(gls_converter* cv, Plane<S, 4> img, float exposure, gls_ycbcr_nlf* out,
                                  cudaStream_t s) {
    GLS_TRY(cv->nlf_scratch.ensure_zeroed(nlf_scratch_bytes() + sizeof(gls_raw_nlf), s));
    GLS_TRY(cv->nlf_stats.ensure(size_t(img.w) * img.h * 4 * sizeof(float)));
    auto* dres = reinterpret_cast<gls_raw_nlf*>(static_cast<char*>(cv->nlf_scratch.p) + nlf_scratch_bytes());
    {
        KScope k(cv->prof, KC_NLF, s, 0);
        cv->prof.launches[KC_NLF] += launch_measure_ycc_nlf<S>(img, plane<float, 4>(cv->nlf_stats, img.w, img.h),
                                                               exposure, cv->nlf_scratch.p, dres, s);
    }
    cv->nlf_sw = img.w;
    cv->nlf_sh = img.h;
    gls_raw_nlf r{};
    GLS_TRY(nlf_result(cv, &r, s));
    for (int c = 0; c < 3; c++) {
        out->a[c] = r.a[c];
        out->b[c] = r.b[c];
    }
    return GLS_OK;
}

template <class S>
static gls_status pyramid_run(gls_converter* cv, Pipeline<S>& P, Plane<S, 4> img0, Plane<S, 2> grad0,
                              const gls_demosaic_params* p, uint32_t flags, cudaStream_t s, bool build_only = false) {
    const int L = p->levels;
    const int W = img0.w, H = img0.h;
    Plane<S, 4> img[GLS_MAX_LEVELS];
    Plane<S, 2> grd[GLS_MAX_LEVELS];
    img[0] = img0;
    grd[0] = grad0;
    for (int i = 1; i < L; i++) {  // Gaussian pyramid, pyramid_processor.cpp:103-120
        img[i] = plane<S, 4>(P.img[i], W >> i, H >> i);
        grd[i] = plane<S, 2>(P.gradp[i], W >> i, H >> i);
        KScope k(cv->prof, KC_DOWNSAMPLE, s);
        launch_downsample_pair<S>(img[i - 1], img[i], grd[i - 1], grd[i], s);
    }
    if (build_only) return GLS_OK;  // the levels run in the persistent batch kernel
    gls_demosaic_params measured;
    if (cv->calibrate) {  // each level's model, measured before the denoise (pyramid_processor.cpp:113-117)
        measured = *p;
        for (int i = 0; i < L; i++) {
            GLS_TRY(measure_ycc_nlf<S>(cv, img[i], p->exposure_multiplier, &measured.pyramid_nlf[i], s));
            cv->nlf_pyr[i] = measured.pyramid_nlf[i];
        }
        cv->nlf_levels = L;
        p = &measured;
    }
    double* acc = static_cast<double*>(P.acc.p);
    float* basis = static_cast<float*>(P.basis.p);
    int* status = static_cast<int*>(P.status.p);
    for (int i = L - 1; i >= 0; i--) {  // coarse to fine, pyramid_processor.cpp:123-168
        const gls_denoise_params& dp = p->denoise[i];
        const int wi = W >> i, hi = H >> i;
        Plane<S, 4> layer = img[i];
        if (i < L - 1) {
            SubtractArgs sa;
            sa.luma_weight = 1.f;  // lumaDenoiseWeight, pyramid_processor.cpp:93
            sa.sharpening = dp.sharpening;
            sa.nlf_a = p->pyramid_nlf[i].a[0] * dp.luma;
            sa.nlf_b = p->pyramid_nlf[i].b[0] * dp.luma;
            layer = plane<S, 4>(P.layer, wi, hi);
            KScope k(cv->prof, KC_SUBTRACT, s);
            launch_subtract_noise<S>(img[i], img[i + 1], plane<S, 4>(P.den[i + 1], W >> (i + 1), H >> (i + 1)), grd[i],
                                     layer, sa, s);
        }
        const int n_patches = (wi / 8) * (hi / 8);
        const int n_blocks = pca_cov_rows(wi, hi);
        double* part = acc + P.acc_off[i];
        {
            KScope k(cv->prof, KC_PCA_COV, s, n_blocks > 0 ? 1 : 0);
            launch_pca_cov<S>(layer, part, s);
        }
        if (flags & GLS_HOST_PCA) {
            P.host_acc.resize(size_t(kPcaAcc) * std::max(1, n_blocks));
            P.host_basis.resize(200);
            if (n_blocks > 0)
                GLS_CUDA(cudaMemcpyAsync(P.host_acc.data(), part, sizeof(double) * kPcaAcc * n_blocks,
                                         cudaMemcpyDeviceToHost, s));
            GLS_CUDA(cudaStreamSynchronize(s));  // the reference's per-level wait, pyramid_processor.cpp:148
            host_pca_basis(P.host_acc.data(), n_blocks, n_patches, P.host_basis.data());
            GLS_CUDA(cudaMemcpyAsync(basis + i * 200, P.host_basis.data(), sizeof(float) * 200,
                                     cudaMemcpyHostToDevice, s));
            GLS_CUDA(cudaStreamSynchronize(s));
        } else {
            KScope k(cv->prof, KC_PCA_EIGEN, s);
            launch_pca_eigen(part, n_blocks, n_patches, basis + i * 200, status + i, s);
        }
        Plane<S, 8> pcap = plane<S, 8>(P.pca, wi, hi);
        if (!is_half<S>::value) {  // the FP16 path projects inside the block-matching kernel
            KScope k(cv->prof, KC_PCA_PROJECT, s);
            launch_pca_project<S>(layer, basis + i * 200, pcap, s);
        }
        BlockMatchArgs ba;
        for (int c = 0; c < 3; c++) {
            ba.var_a[c] = p->pyramid_nlf[i].a[c];
            ba.var_b[c] = p->pyramid_nlf[i].b[c];
        }
        ba.tm[0] = dp.luma;
        ba.tm[1] = dp.chroma;
        ba.tm[2] = dp.chroma;
        ba.chroma_boost = dp.chroma_boost;
        ba.gradient_boost = dp.gradient_boost;
        ba.gradient_threshold = dp.gradient_threshold;
        ba.lsc = p->lens_shading_correction;
        ba.tensor = flags & GLS_BM_TENSOR;
        if (!is_half<S>::value && cv->keep_nc) {
            GLS_TRY(P.nc[i].ensure(size_t(wi) * hi * sizeof(float)));
            ba.nc_out = static_cast<float*>(P.nc[i].p);
        }
        KScope k(cv->prof, KC_BLOCK_MATCH, s);
        launch_block_match<S>(layer, grd[i], pcap, basis + i * 200, plane<S, 4>(P.den[i], wi, hi), ba, s);
    }
    GLS_CUDA(cudaGetLastError());
    cv->last_levels = L;
    return GLS_OK;
}

// A batch slot's host copies on their own streams: the next frame's raw
// upload waits only until the previous frame's scale_raw has read the raw
// staging buffer, and its output transform only until the previous
// frame's download has emptied the output staging buffer.
struct SlotCopies {
    cudaStream_t in, out;
    cudaEvent_t raw_free, raw_ready, out_ready, out_free;
};

template <class S, class O>
static gls_status finish_output(gls_converter* cv, Plane<S, 4> src, bool transform, const float* m, OutTarget<O>& t,
                                cudaStream_t s, const SlotCopies* cp = nullptr, const PostArgs<S>* post = nullptr) {
    if (cp && t.copy_to_host) GLS_CUDA(cudaStreamWaitEvent(s, cp->out_free, 0));
    if (post) {  // the display post-processing writes the output
        KScope k(cv->prof, KC_POST, s, 0);
        cv->prof.launches[KC_POST] += launch_post<S, O>(*post, t.plane, s);
    } else {
        KScope k(cv->prof, KC_OUTPUT, s);
        if (transform) {
            Mat3Args ma;
            std::memcpy(ma.m, m, sizeof(ma.m));
            launch_transform<S, O>(src, t.plane, ma, s);
        } else {
            launch_convert4<S, O>(src, t.plane, s);
        }
    }
    GLS_CUDA(cudaGetLastError());
    if (t.copy_to_host) {
        const size_t row = size_t(t.plane.w) * 4 * sizeof(O);
        cudaStream_t cs = s;
        if (cp) {
            GLS_CUDA(cudaEventRecord(cp->out_ready, s));
            GLS_CUDA(cudaStreamWaitEvent(cp->out, cp->out_ready, 0));
            cs = cp->out;
        }
        GLS_CUDA(cudaMemcpy2DAsync(t.host, t.host_stride, t.plane.p, t.plane.pitch * sizeof(O), row, t.plane.h,
                                   cudaMemcpyDeviceToHost, cs));
        if (cp) GLS_CUDA(cudaEventRecord(cp->out_free, cp->out));
    }
    return GLS_OK;
}

template <class S, class O>
static gls_status make_target(Pipeline<S>& P, gls_image_view* out, int w, int h, bool host_io, OutTarget<O>& t) {
    DevBuf& own = sizeof(O) == 4 ? P.out_f32 : P.out_f16;
    if (!out->data || host_io) {
        GLS_TRY(own.ensure(size_t(w) * h * 4 * sizeof(O)));
        t.plane = plane<O, 4>(own, w, h);
        if (out->data) {
            t.copy_to_host = true;
            t.host = out->data;
            t.host_stride = out->stride_bytes ? out->stride_bytes : size_t(w) * 4 * sizeof(O);
            if (t.host_stride < size_t(w) * 4 * sizeof(O)) return set_error(GLS_ERR_INVALID_ARG, "output stride too small");
        } else {
            out->data = own.p;
            out->width = w;
            out->height = h;
            out->channels = 4;
            out->stride_bytes = size_t(w) * 4 * sizeof(O);
        }
    } else {
        const size_t stride = out->stride_bytes ? out->stride_bytes : size_t(w) * 4 * sizeof(O);
        if (stride % (4 * sizeof(O)) || stride < size_t(w) * 4 * sizeof(O) || (uintptr_t(out->data) % (4 * sizeof(O))))
            return set_error(GLS_ERR_INVALID_ARG, "device output must be %zu-byte aligned with a matching stride",
                             4 * sizeof(O));
        t.plane = Plane<O, 4>{static_cast<O*>(out->data), w, h, stride / sizeof(O)};
    }
    return GLS_OK;
}

// crossDenoiseRawRGBAImage arguments (raw_converter.cpp:195-202)
static RawDenoiseArgs raw_denoise_args(const gls_demosaic_params* p, bool fast) {
    RawDenoiseArgs ra;
    ra.pattern = p->bayer_pattern;
    for (int c = 0; c < 4; c++) ra.var[c] = p->raw_nlf.b[c];
    ra.strength = p->raw_denoise_strength;
    ra.fast = fast ? 1 : 0;
    return ra;
}

// demosaic arguments: getRawVariance (demosaic.hpp:186-193), green the mean
// of G and G2; cam -> YCbCr when the image goes on to the denoiser
static DemosaicArgs demosaic_args(const gls_demosaic_params* p, bool transform) {
    DemosaicArgs da;
    da.pattern = p->bayer_pattern;
    da.rv0 = p->raw_nlf.a[0];
    da.rv1 = p->raw_nlf.b[0];
    da.gv0 = (p->raw_nlf.a[1] + p->raw_nlf.a[3]) / 2;
    da.gv1 = (p->raw_nlf.b[1] + p->raw_nlf.b[3]) / 2;
    da.bv0 = p->raw_nlf.a[2];
    da.bv1 = p->raw_nlf.b[2];
    da.transform = transform ? 1 : 0;
    float c2y[9], y2c[9];
    cam_ycbcr(p->rgb_cam, p->xyz_rgb, c2y, y2c);
    std::memcpy(da.m, c2y, sizeof(c2y));
    return da;
}

// Stages of a frame: the whole frame, or (persistent batches) the front end
// and the pyramid's images only, or the output only (after the levels).
enum { STAGE_ALL = 0, STAGE_FRONT = 1, STAGE_OUTPUT = 2 };

template <class S>
static gls_status demosaic_run(gls_converter* cv, const uint16_t* raw, int w, int h, size_t stride_bytes,
                               const gls_demosaic_params* p, uint32_t flags, gls_image_view* out, cudaStream_t s,
                               int slot = 0, const SlotCopies* cp = nullptr, int stage = STAGE_ALL,
                               Pipeline<S>* use = nullptr) {
    Pipeline<S>& P = use ? *use
                         : *reinterpret_cast<Pipeline<S>*>(is_half<S>::value ? (void*)&cv->p16s[slot]
                                                                            : (void*)&cv->p32s[slot]);
    const bool host_io = flags & GLS_HOST_IO;
    const bool denoise = flags & GLS_DENOISE;
    GLS_TRY(P.ensure(w, h, p->levels));
    if (stage == STAGE_OUTPUT) {  // the levels are done: transformImage(YCbCr -> cam) of level 0
        float c2y[9], y2c[9];
        cam_ycbcr(p->rgb_cam, p->xyz_rgb, c2y, y2c);
        const Plane<S, 4> den0 = plane<S, 4>(P.den[0], w, h);
        if (out->dtype == GLS_F16) {
            OutTarget<__half> t;
            GLS_TRY(make_target<S, __half>(P, out, w, h, host_io, t));
            return finish_output<S, __half>(cv, den0, true, y2c, t, s, cp, nullptr);
        }
        out->dtype = GLS_F32;
        OutTarget<float> t;
        GLS_TRY(make_target<S, float>(P, out, w, h, host_io, t));
        return finish_output<S, float>(cv, den0, true, y2c, t, s, cp, nullptr);
    }

    // raw input
    const uint16_t* rawp = raw;
    size_t raw_pitch = stride_bytes / 2;
    if (host_io) {
        if (cp) GLS_CUDA(cudaStreamWaitEvent(cp->in, cp->raw_free, 0));
        GLS_CUDA(cudaMemcpy2DAsync(P.raw.p, size_t(w) * 2, raw, stride_bytes, size_t(w) * 2, h,
                                   cudaMemcpyHostToDevice, cp ? cp->in : s));
        if (cp) {
            GLS_CUDA(cudaEventRecord(cp->raw_ready, cp->in));
            GLS_CUDA(cudaStreamWaitEvent(s, cp->raw_ready, 0));
        }
        rawp = static_cast<const uint16_t*>(P.raw.p);
        raw_pitch = size_t(w);
    } else if ((uintptr_t(raw) & 3) || (stride_bytes & 3)) {
        return set_error(GLS_ERR_INVALID_ARG, "device raw input must be 4-byte aligned with a 4-byte multiple stride");
    }

    Plane<S, 1> scaled = plane<S, 1>(P.scaled, w, h);
    Plane<S, 2> grad = plane<S, 2>(P.grad, w, h);

    // scaleRawData, raw_converter.cpp:179-183
    ScaleArgs sa;
    sa.pattern = p->bayer_pattern;
    sa.black = int(lroundf(p->black_level));
    for (int c = 0; c < 4; c++) sa.k[c] = float(double(p->scale_mul[c]) * 0.9 / 65535.0);
    sa.lsc = p->lens_shading_correction;
    sa.cx = float(w / 2);
    sa.cy = float(h / 2);
    {
        volatile float cx2 = sa.cx * sa.cx, cy2 = sa.cy * sa.cy;
        volatile float ss = cx2 + cy2;
        sa.clen = sqrtf(ss);
    }
    {
        KScope k(cv->prof, KC_SCALE, s);
        launch_scale_raw<S>(rawp, raw_pitch, scaled, sa, s);
    }
    if (cp && host_io) GLS_CUDA(cudaEventRecord(cp->raw_free, s));  // the raw staging buffer is read

    // calibrateFromImage: the raw model measured on the scaled frame, the
    // high-noise branch off (raw_converter.cpp:160, 188-189)
    gls_demosaic_params calibrated;
    if (cv->calibrate) {
        calibrated = *p;
        calibrated.high_noise_image = 0;
        GLS_TRY(measure_raw_nlf<S>(cv, scaled, p->bayer_pattern, p->exposure_multiplier, &calibrated.raw_nlf, s));
        cv->nlf_raw = calibrated.raw_nlf;
        cv->nlf_levels = 0;
        p = &calibrated;
    }

    // rawImageSobel + sampledConvolutionSobel, raw_converter.cpp:185-193
    BlurArgs ba;
    float taps[3 * kMaxTaps];
    const int n1 = gaussian_taps(1.5f, taps, kMaxTaps);
    const int n2 = gaussian_taps(4.5f, taps + 3 * n1, kMaxTaps - n1);
    if (n1 <= 0 || n2 <= 0) return set_error(GLS_ERR_INVALID_ARG, "blur tap table overflow");
    ba.n1 = n1;
    ba.n2 = n2;
    for (int t = 0; t < n1 + n2; t++) {
        ba.w[t] = taps[3 * t];
        const float fdx = floorf(taps[3 * t + 1]), fdy = floorf(taps[3 * t + 2]);
        ba.ix[t] = int(fdx);
        ba.iy[t] = int(fdy);
        ba.fx[t] = taps[3 * t + 1] - fdx;
        ba.fy[t] = taps[3 * t + 2] - fdy;
    }
    // the green raw variance (getRawVariance, demosaic.hpp:186-193)
    ba.var0 = (p->raw_nlf.a[1] + p->raw_nlf.a[3]) / 2;
    ba.var1 = (p->raw_nlf.b[1] + p->raw_nlf.b[3]) / 2;
    ba.inv_sqrt45 = 1.0f / sqrtf(4.5f);
    {
        KScope k(cv->prof, KC_SOBEL_BLUR, s);
        launch_sobel_blur<S>(scaled, grad, ba, s);
    }

    // high-noise raw branch, raw_converter.cpp:195-202
    if (denoise && p->high_noise_image) {
        if (!is_half<S>::value && cv->keep_nc) {  // the adjoint's front-end tangents read it
            GLS_TRY(P.scaled0.ensure(size_t(w) * h * sizeof(S)));
            GLS_CUDA(cudaMemcpyAsync(P.scaled0.p, P.scaled.p, size_t(w) * h * sizeof(S), cudaMemcpyDeviceToDevice, s));
        }
        const RawDenoiseArgs ra = raw_denoise_args(p, is_half<S>::value);
        KScope k(cv->prof, KC_RAW_DENOISE, s, 2);
        launch_raw_denoise<S>(scaled, grad, plane<S, 4>(P.quad, w / 2, h / 2), ra, s);
    }

    // demosaic + blendHighlights (+ cam -> YCbCr), raw_converter.cpp:204-214
    float c2y[9], y2c[9];
    cam_ycbcr(p->rgb_cam, p->xyz_rgb, c2y, y2c);
    const DemosaicArgs da = demosaic_args(p, denoise);
    Plane<S, 4> A = plane<S, 4>(P.A, w, h);
    {
        KScope k(cv->prof, KC_DEMOSAIC, s);
        launch_demosaic<S>(scaled, grad, A, da, s);
    }
    GLS_CUDA(cudaGetLastError());

    Plane<S, 4> final_src = A;
    if (denoise) {
        // RawConverter::denoise, raw_converter.cpp:70-116
        Plane<S, 4> B = plane<S, 4>(P.B, w, h);
        {
            KScope k(cv->prof, KC_DESPECKLE, s);
            launch_despeckle<S>(A, B, p->pyramid_nlf[0].a[0], p->pyramid_nlf[0].b[0], s);
        }
        GLS_TRY(pyramid_run<S>(cv, P, B, grad, p, flags, s, stage == STAGE_FRONT));
        if (stage == STAGE_FRONT) return GLS_OK;
        final_src = plane<S, 4>(P.den[0], w, h);
        if (cv->calibrate)  // the post-processing reads the measured level-0 model
            for (int i = 0; i < p->levels; i++) calibrated.pyramid_nlf[i] = cv->nlf_pyr[i];
    }
    // display post-processing (raw_converter.cpp:80-116, 231-244)
    PostArgs<S> pa{};
    const bool post = flags & GLS_POSTPROCESS;
    if (post) {
        pa.params = p;
        std::memcpy(pa.y2c, y2c, sizeof(pa.y2c));
        pa.denoise = denoise;
        if (denoise)
            for (int l = 0; l < 5; l++) pa.den[l] = plane<S, 4>(P.den[l], w >> l, h >> l);
        pa.rgb = A;
        pa.grad2 = grad;
        pa.raw = rawp;
        GLS_TRY(P.post_hist.ensure_zeroed(256 * sizeof(uint32_t), s));
        GLS_TRY(P.post_stats.ensure(sizeof(PostStats)));
        GLS_TRY(P.post_perm.ensure(kNoiseSize * sizeof(int)));
        GLS_TRY(P.post_gtab.ensure(kNoiseSize * 2 * sizeof(float)));
        GLS_TRY(P.post_ab.ensure(post_ab_bytes(w, h)));
        pa.hist = static_cast<uint32_t*>(P.post_hist.p);
        pa.stats = static_cast<PostStats*>(P.post_stats.p);
        pa.perm = static_cast<int*>(P.post_perm.p);
        pa.grad_tab = static_cast<float*>(P.post_gtab.p);
        pa.ab = static_cast<float2*>(P.post_ab.p);
    }
    // transformImage(YCbCr -> cam), raw_converter.cpp:219
    if (out->dtype == GLS_F16) {
        OutTarget<__half> t;
        GLS_TRY(make_target<S, __half>(P, out, w, h, host_io, t));
        GLS_TRY(finish_output<S, __half>(cv, final_src, denoise, y2c, t, s, cp, post ? &pa : nullptr));
    } else {
        out->dtype = GLS_F32;
        OutTarget<float> t;
        GLS_TRY(make_target<S, float>(P, out, w, h, host_io, t));
        GLS_TRY(finish_output<S, float>(cv, final_src, denoise, y2c, t, s, cp, post ? &pa : nullptr));
    }
    if (slot == 0) {
        cv->last_storage = is_half<S>::value ? GLS_F16 : GLS_F32;
        cv->last_w = w;
        cv->last_h = h;
        cv->last_denoise = denoise;
        // a single frame returns with its result (the reference is
        // synchronous); a batch synchronises once, after its join
        if (!cp && (host_io || (flags & GLS_SYNC))) GLS_CUDA(cudaStreamSynchronize(s));
    }
    return GLS_OK;
}

template <class S>
static gls_status pyramid_only(gls_converter* cv, const gls_image_view* ycc, const gls_image_view* gradient,
                               const gls_demosaic_params* p, uint32_t flags, gls_image_view* out, cudaStream_t s) {
    Pipeline<S>& P = *reinterpret_cast<Pipeline<S>*>(is_half<S>::value ? (void*)&cv->p16 : (void*)&cv->p32);
    const int w = ycc->width, h = ycc->height;
    const bool host_io = flags & GLS_HOST_IO;
    GLS_TRY(P.ensure(w, h, p->levels));
    Plane<S, 4> B = plane<S, 4>(P.B, w, h);
    Plane<S, 2> grad = plane<S, 2>(P.grad, w, h);
    {
        KScope k(cv->prof, KC_VIEW_IN, s, 2);
        GLS_TRY(view_to_plane<S, 4>(ycc, host_io, P.stage_in, B, s));
        GLS_TRY(view_to_plane<S, 2>(gradient, host_io, P.stage_grad, grad, s));
    }
    GLS_TRY(pyramid_run<S>(cv, P, B, grad, p, flags, s));
    Plane<S, 4> den0 = plane<S, 4>(P.den[0], w, h);
    if (out->dtype == GLS_F16) {
        OutTarget<__half> t;
        GLS_TRY(make_target<S, __half>(P, out, w, h, host_io, t));
        GLS_TRY(finish_output<S, __half>(cv, den0, false, nullptr, t, s));
    } else {
        out->dtype = GLS_F32;
        OutTarget<float> t;
        GLS_TRY(make_target<S, float>(P, out, w, h, host_io, t));
        GLS_TRY(finish_output<S, float>(cv, den0, false, nullptr, t, s));
    }
    cv->last_storage = is_half<S>::value ? GLS_F16 : GLS_F32;
    cv->last_w = w;
    cv->last_h = h;
    cv->last_denoise = true;
    if (host_io || (flags & GLS_SYNC)) GLS_CUDA(cudaStreamSynchronize(s));
    return GLS_OK;
}

}  // namespace gls

// ============================================================== C ABI
namespace gls {

// The reverse sweep over the FP32 pipeline's retained planes (slot 0): the
// loss head, then per level fine to coarse block matching transposed and,
// below the coarsest level, the reconstruct step transposed into the next
// level's denoised image. grad receives GLS_ADJ_NPARAMS values.
// The reverse sweep over the FP32 forward's retained planes (slot 0).
// Head: the MSE of the output RGB against `target` (loss and its
// gradient), or, with target NULL, the given cotangent g_out3 (3 ch,
// tightly packed) of the denoised YCbCr. front_end: add the raw front
// end's tangents (parameters 30, 31; else 0).
static gls_status adjoint_run(gls_converter* cv, const gls_demosaic_params* p, const float* target, int tstride,
                              const float* g_out3, bool front_end, double* loss, float* grad, cudaStream_t s) {
    Pipeline<float>& P = cv->p32s[0];
    const int W = P.W, H = P.H, L = p->levels;
    const size_t n = size_t(W) * H;
    GLS_TRY(cv->adj_gden[0].ensure(n * 3 * sizeof(float)));
    GLS_TRY(cv->adj_gden[1].ensure(n * 3 * sizeof(float)));
    GLS_TRY(cv->adj_rec.ensure(n * 12 * sizeof(float)));
    GLS_TRY(cv->adj_glayer.ensure(n * 4 * sizeof(float)));
    GLS_TRY(cv->adj_gpca.ensure(n * 8 * sizeof(float)));
    GLS_TRY(cv->adj_gup.ensure(n * 3 * sizeof(float)));
    // dL/d img_l for every level (3 ch), and the front-end tangent scratch
    std::vector<size_t> gimg_off(L + 1, 0);
    for (int i = 0; i < L; i++) gimg_off[i + 1] = gimg_off[i] + size_t(W >> i) * (H >> i) * 3;
    GLS_TRY(cv->adj_gimg.ensure(gimg_off[L] * sizeof(float)));
    GLS_TRY(cv->adj_gp1.ensure(n * 3 * sizeof(float)));
    const int jvp_blocks = front_jvp_blocks(W, H);
    if (front_end) {
        GLS_TRY(cv->adj_jvp.ensure(front_jvp_scratch_bytes(W, H)));
        GLS_TRY(cv->adj_jvp_part.ensure(size_t(jvp_blocks) * 2 * sizeof(float)));
    }
    float* gimg = static_cast<float*>(cv->adj_gimg.p);
    GLS_CUDA(cudaMemsetAsync(gimg, 0, gimg_off[L] * sizeof(float), s));
    std::vector<size_t> bm_off(L), sn_off(L);
    size_t parts = 0;
    for (int i = 0; i < L; i++) {
        bm_off[i] = parts;
        parts += size_t(adjoint_blocks(W >> i, H >> i)) * 6;
        sn_off[i] = parts;
        if (i < L - 1) parts += size_t(adjoint_sn_blocks(W >> i, H >> i)) * 2;
    }
    const int head_blocks = adjoint_sn_blocks(W, H);
    GLS_TRY(cv->adj_part.ensure(std::max<size_t>(parts, 1) * sizeof(float)));
    GLS_TRY(cv->adj_loss.ensure(size_t(head_blocks) * sizeof(double)));
    float* part = static_cast<float*>(cv->adj_part.p);

    float c2y[9], y2c[9];
    cam_ycbcr(p->rgb_cam, p->xyz_rgb, c2y, y2c);
    AdjointHeadArgs ha;
    std::memcpy(ha.m, y2c, sizeof(y2c));
    ha.inv_n = float(1.0 / (3.0 * double(n)));
    float* gcur = static_cast<float*>(cv->adj_gden[0].p);
    float* gnext = static_cast<float*>(cv->adj_gden[1].p);
    if (target)
        launch_adj_head(static_cast<const float*>(P.den[0].p), target, tstride, W, H, ha, gcur,
                        static_cast<double*>(cv->adj_loss.p), s);
    else
        GLS_CUDA(cudaMemcpyAsync(gcur, g_out3, n * 3 * sizeof(float), cudaMemcpyDeviceToDevice, s));
    for (int i = 0; i < L; i++) {
        const int wi = W >> i, hi = H >> i;
        const gls_denoise_params& dp = p->denoise[i];
        const float* img_i = static_cast<const float*>(i == 0 ? P.B.p : P.img[i].p);
        const float* grd = static_cast<const float*>(i == 0 ? P.grad.p : P.gradp[i].p);
        const float* basis = static_cast<const float*>(P.basis.p) + i * 200;
        // the level's reconstructed layer, recomputed from the retained
        // pyramid (the forward keeps one layer buffer for all levels): the
        // same kernel on the same inputs, so the same bits
        const float* layer = img_i;
        if (i < L - 1) {
            SubtractArgs ra;
            ra.luma_weight = 1.f;
            ra.sharpening = dp.sharpening;
            ra.nlf_a = p->pyramid_nlf[i].a[0] * dp.luma;
            ra.nlf_b = p->pyramid_nlf[i].b[0] * dp.luma;
            const int cw = W >> (i + 1), ch = H >> (i + 1);
            launch_subtract_noise<float>(Plane<float, 4>{const_cast<float*>(img_i), wi, hi, size_t(wi) * 4},
                                         plane<float, 4>(P.img[i + 1], cw, ch), plane<float, 4>(P.den[i + 1], cw, ch),
                                         Plane<float, 2>{const_cast<float*>(grd), wi, hi, size_t(wi) * 2},
                                         plane<float, 4>(P.layer, wi, hi), ra, s);
            layer = static_cast<const float*>(P.layer.p);
        }
        launch_pca_project<float>(Plane<float, 4>{const_cast<float*>(layer), wi, hi, size_t(wi) * 4}, basis,
                                  plane<float, 8>(P.pca, wi, hi), s);
        AdjointLevelArgs la{};
        la.w = wi;
        la.h = hi;
        la.den = static_cast<const float*>(P.den[i].p);
        la.nc = static_cast<const float*>(P.nc[i].p);
        la.layer = layer;
        la.grad = grd;
        la.pca = static_cast<const float*>(P.pca.p);
        la.basis = basis;
        la.g_den = gcur;
        la.rec = static_cast<float*>(cv->adj_rec.p);
        la.g_layer = static_cast<float*>(cv->adj_glayer.p);
        la.g_pca = static_cast<float*>(cv->adj_gpca.p);
        la.part = part + bm_off[i];
        for (int c = 0; c < 3; c++) {
            la.var_a[c] = p->pyramid_nlf[i].a[c];
            la.var_b[c] = p->pyramid_nlf[i].b[c];
        }
        la.tm[0] = dp.luma;
        la.tm[1] = dp.chroma;
        la.tm[2] = dp.chroma;
        la.chroma_boost = dp.chroma_boost;
        la.gradient_boost = dp.gradient_boost;
        la.gradient_threshold = dp.gradient_threshold;
        launch_bm_bwd(la, s);
        if (i < L - 1) {
            AdjointSnArgs sa{};
            sa.w = wi;
            sa.h = hi;
            sa.cw = W >> (i + 1);
            sa.ch = H >> (i + 1);
            sa.rx = float(sa.cw) / float(wi);
            sa.ry = float(sa.ch) / float(hi);
            sa.in = img_i;
            sa.coarse = static_cast<const float*>(P.img[i + 1].p);
            sa.coarse_den = static_cast<const float*>(P.den[i + 1].p);
            sa.grad = grd;
            sa.g_layer = la.g_layer;
            sa.g_up = static_cast<float*>(cv->adj_gup.p);
            sa.g_coarse_den = gnext;
            sa.part = part + sn_off[i];
            sa.luma_weight = 1.f;
            sa.sharpening = dp.sharpening;
            sa.nlf_a = p->pyramid_nlf[i].a[0] * dp.luma;
            sa.nlf_b = p->pyramid_nlf[i].b[0] * dp.luma;
            sa.g_in = gimg + gimg_off[i];
            sa.g_p1 = static_cast<float*>(cv->adj_gp1.p);
            sa.g_coarse_img = gimg + gimg_off[i + 1];
            launch_sn_bwd(sa, s);
            std::swap(gcur, gnext);
        } else {  // the coarsest level denoises its image itself
            launch_add_layer_grad(la.g_layer, gimg + gimg_off[i], wi, hi, s);
        }
    }
    // img_{l+1} = down(img_l): push dL/d img down to the despeckled image
    for (int i = L - 2; i >= 0; i--)
        launch_down_bwd(gimg + gimg_off[i + 1], W >> (i + 1), H >> (i + 1), gimg + gimg_off[i], W >> i, H >> i, s);
    // the raw front end's tangents along theta30 / theta31, dotted with it
    if (front_end) {
        FrontJvpArgs fj;
        fj.w = W;
        fj.h = H;
        fj.scaled = static_cast<const float*>(P.scaled.p);
        fj.scaled0 = static_cast<const float*>(P.scaled0.p);
        fj.quad = static_cast<const float*>(P.quad.p);
        fj.grad = static_cast<const float*>(P.grad.p);
        fj.high_noise = p->high_noise_image ? 1 : 0;
        fj.raw = raw_denoise_args(p, false);
        fj.dm = demosaic_args(p, true);
        fj.despeckle_va = p->pyramid_nlf[0].a[0];
        fj.despeckle_vb = p->pyramid_nlf[0].b[0];
        fj.g_ds = gimg;
        fj.scratch = cv->adj_jvp.p;
        fj.part = static_cast<float*>(cv->adj_jvp_part.p);
        launch_front_jvp(fj, s);
    }
    cv->adj_gimg_w = W;
    cv->adj_gimg_h = H;
    GLS_CUDA(cudaGetLastError());
    std::vector<float> hp(parts), hj(front_end ? size_t(jvp_blocks) * 2 : 0);
    std::vector<double> hl(target ? head_blocks : 0);
    if (parts) GLS_CUDA(cudaMemcpyAsync(hp.data(), part, parts * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (!hj.empty())
        GLS_CUDA(cudaMemcpyAsync(hj.data(), cv->adj_jvp_part.p, hj.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (!hl.empty())
        GLS_CUDA(cudaMemcpyAsync(hl.data(), cv->adj_loss.p, hl.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    GLS_CUDA(cudaStreamSynchronize(s));
    double g[GLS_ADJ_NPARAMS] = {};
    for (int i = 0; i < L; i++) {
        const int nb = adjoint_blocks(W >> i, H >> i);
        double t[6] = {0, 0, 0, 0, 0, 0};
        for (int b = 0; b < nb; b++)
            for (int k = 0; k < 6; k++) t[k] += hp[bm_off[i] + size_t(b) * 6 + k];
        g[GLS_ADJ_LUMA + i] += t[0];
        g[GLS_ADJ_CHROMA + i] += t[1];
        g[GLS_ADJ_NLF_AY + i] += t[2];
        g[GLS_ADJ_NLF_BY + i] += t[3];
        g[GLS_ADJ_NLF_AC + i] += t[4];
        g[GLS_ADJ_NLF_BC + i] += t[5];
        if (i < L - 1) {  // nlf_a = A_Y luma, nlf_b = B_Y luma
            const int ns = adjoint_sn_blocks(W >> i, H >> i);
            double ga = 0, gb = 0;
            for (int b = 0; b < ns; b++) {
                ga += hp[sn_off[i] + size_t(b) * 2];
                gb += hp[sn_off[i] + size_t(b) * 2 + 1];
            }
            const double luma = p->denoise[i].luma;
            g[GLS_ADJ_NLF_AY + i] += ga * luma;
            g[GLS_ADJ_NLF_BY + i] += gb * luma;
            g[GLS_ADJ_LUMA + i] += ga * p->pyramid_nlf[i].a[0] + gb * p->pyramid_nlf[i].b[0];
        }
    }
    double lsum = 0;
    for (double v : hl) lsum += v;
    if (loss) *loss = lsum / (3.0 * double(n));
    for (size_t b = 0; b < hj.size() / 2; b++) {
        g[GLS_ADJ_RAW_GREEN_A] += hj[b * 2];
        g[GLS_ADJ_RAW_GREEN_B] += hj[b * 2 + 1];
    }
    for (int k = 0; k < GLS_ADJ_NPARAMS; k++) grad[k] = float(g[k]);
    return GLS_OK;
}

}  // namespace gls

namespace gls {

// Signature of a batch for graph replay: pointers, sizes, strides, output
// views, flags and the bytes of every parameter block (kernel arguments are
// baked into the graph). Empty when an output is converter-owned.
static std::vector<uint64_t> batch_key(const gls_frame_desc* frames, int n, uint32_t flags) {
    std::vector<uint64_t> k;
    k.push_back(uint64_t(n));
    k.push_back(flags);
    for (int i = 0; i < n; i++) {
        const gls_frame_desc& f = frames[i];
        if (!f.out.data) return {};
        k.push_back(uint64_t(uintptr_t(f.raw)));
        k.push_back((uint64_t(uint32_t(f.width)) << 32) | uint32_t(f.height));
        k.push_back(f.raw_stride_bytes);
        k.push_back(uint64_t(uintptr_t(f.out.data)));
        k.push_back((uint64_t(uint32_t(f.out.dtype)) << 32) | uint32_t(f.out.channels));
        k.push_back(f.out.stride_bytes);
        uint64_t h = 1469598103934665603ull;  // FNV-1a over the parameter block
        const unsigned char* b = reinterpret_cast<const unsigned char*>(f.params);
        for (size_t j = 0; j < sizeof(gls_demosaic_params); j++) h = (h ^ b[j]) * 1099511628211ull;
        k.push_back(h);
    }
    return k;
}

// The work list of a persistent batch: a descriptor per (frame, level) and
// the tasks, level by level from the coarsest, all frames' reconstruct /
// covariance / eigen-solve tasks of a level before their block-matching
// tiles (the order the kernel's dependency waits rely on).
static gls_status persistent_plan(gls_converter* conv, const gls_frame_desc* frames, int n) {
    std::vector<PLevel> lv;
    std::vector<int> first(n);  // descriptor index of each frame's level 0
    int max_levels = 0;
    for (int f = 0; f < n; f++) {
        const gls_demosaic_params* p = frames[f].params;
        Pipeline<__half>& P = *conv->pframes[f];
        const int W = frames[f].width, H = frames[f].height, L = p->levels;
        max_levels = std::max(max_levels, L);
        first[f] = int(lv.size());
        for (int i = 0; i < L; i++) {
            const int wi = W >> i, hi = H >> i;
            PLevel d{};
            d.img = i == 0 ? plane<__half, 4>(P.B, W, H) : plane<__half, 4>(P.img[i], wi, hi);
            d.grad = i == 0 ? plane<__half, 2>(P.grad, W, H) : plane<__half, 2>(P.gradp[i], wi, hi);
            d.layer = i < L - 1 ? plane<__half, 4>(P.layer, wi, hi) : d.img;
            d.den = plane<__half, 4>(P.den[i], wi, hi);
            if (i < L - 1) {
                const int cw = W >> (i + 1), ch = H >> (i + 1);
                d.coarse = plane<__half, 4>(P.img[i + 1], cw, ch);
                d.coarse_den = plane<__half, 4>(P.den[i + 1], cw, ch);
                d.rx = float(cw) / float(wi);
                d.ry = float(ch) / float(hi);
            }
            const gls_denoise_params& dp = p->denoise[i];
            d.sa.luma_weight = 1.f;  // lumaDenoiseWeight, pyramid_processor.cpp:93
            d.sa.sharpening = dp.sharpening;
            d.sa.nlf_a = p->pyramid_nlf[i].a[0] * dp.luma;
            d.sa.nlf_b = p->pyramid_nlf[i].b[0] * dp.luma;
            for (int c = 0; c < 3; c++) {
                d.ba.var_a[c] = p->pyramid_nlf[i].a[c];
                d.ba.var_b[c] = p->pyramid_nlf[i].b[c];
            }
            d.ba.tm[0] = dp.luma;
            d.ba.tm[1] = dp.chroma;
            d.ba.tm[2] = dp.chroma;
            d.ba.chroma_boost = dp.chroma_boost;
            d.ba.gradient_boost = dp.gradient_boost;
            d.ba.gradient_threshold = dp.gradient_threshold;
            d.ba.lsc = p->lens_shading_correction;
            d.ba.nc_out = nullptr;
            d.part = static_cast<double*>(P.acc.p) + P.acc_off[i];
            d.basis = static_cast<float*>(P.basis.p) + i * 200;
            d.status = static_cast<int*>(P.status.p) + i;
            d.tiles_x = (wi + 31) / 32;
            d.n_bm = d.tiles_x * ((hi + 31) / 32);
            d.sn_tiles_x = (wi + kPSnTile - 1) / kPSnTile;
            d.n_sn = i < L - 1 ? d.sn_tiles_x * ((hi + kPSnTile - 1) / kPSnTile) : 0;
            d.n_cov = pca_cov_rows(wi, hi);
            d.chunks = pca_cov_chunks(wi, hi);
            d.cov_group = pca_cov_group(d.chunks);
            d.coarser = i < L - 1 ? first[f] + i + 1 : -1;
            // every plane the kernel reads or writes must exist (the front
            // ends, which run before the plan is built, size them)
            if (!d.img.p || !d.grad.p || !d.layer.p || !d.den.p || !P.acc.p || !P.basis.p || !P.status.p ||
                (i < L - 1 && (!d.coarse.p || !d.coarse_den.p)))
                return set_error(GLS_ERR_INVALID_ARG, "persistent plan: frame %d level %d has unallocated planes", f,
                                 i);
            lv.push_back(d);
        }
    }
    std::vector<PTask> tasks;
    auto put = [&](int lev, uint32_t type, int count) {
        for (int k = 0; k < count; k++) tasks.push_back({uint32_t(lev), (type << 30) | uint32_t(k)});
    };
    for (int i = max_levels - 1; i >= 0; i--) {
        for (int f = 0; f < n; f++) {
            if (i >= frames[f].params->levels) continue;
            const int lev = first[f] + i;
            put(lev, PT_SN, lv[lev].n_sn);
            put(lev, PT_COV, lv[lev].n_cov);
            put(lev, PT_EIG, 1);
        }
        for (int f = 0; f < n; f++)
            if (i < frames[f].params->levels) put(first[f] + i, PT_BM, lv[first[f] + i].n_bm);
    }
    GLS_TRY(conv->plan_task_buf.ensure(tasks.size() * sizeof(PTask)));
    GLS_TRY(conv->plan_level_buf.ensure(lv.size() * sizeof(PLevel)));
    GLS_TRY(conv->plan_cnt.ensure(lv.size() * sizeof(PCounters)));
    GLS_TRY(conv->plan_ctl.ensure(2 * sizeof(int)));
    GLS_CUDA(cudaMemcpy(conv->plan_task_buf.p, tasks.data(), tasks.size() * sizeof(PTask), cudaMemcpyHostToDevice));
    GLS_CUDA(cudaMemcpy(conv->plan_level_buf.p, lv.data(), lv.size() * sizeof(PLevel), cudaMemcpyHostToDevice));
    conv->plan_tasks = int(tasks.size());
    conv->plan_levels = int(lv.size());
    return GLS_OK;
}

// Wait limit of the persistent kernel's dependency waits: far above any
// level's duration (a dependency is at most one level of the batch away).
constexpr long long kPersistentWaitNs = 2000000000ll;

// A persistent batch: every frame's front end and pyramid images on the
// slot streams (frames LPT-assigned as in enqueue_batch, each into a
// pyramid of its own), then one launch for every level of every frame,
// then every frame's output transform.
static gls_status persistent_batch(gls_converter* conv, gls_frame_desc* frames, int n, uint32_t flags, cudaStream_t s,
                                   const std::vector<int>& order, const std::vector<int>& slot_of, int nslots,
                                   bool capturing) {
    while (int(conv->pframes.size()) < n) conv->pframes.push_back(std::make_unique<Pipeline<__half>>());
    GLS_CUDA(cudaEventRecord(conv->fork_ev, s));
    for (int k = 0; k < nslots; k++) GLS_CUDA(cudaStreamWaitEvent(conv->slot_stream[k], conv->fork_ev, 0));
    gls_status result = GLS_OK;
    for (int oi = 0; oi < n && result == GLS_OK; oi++) {
        const int i = order[oi];
        gls_frame_desc& f = frames[i];
        result = demosaic_run<__half>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params, flags, &f.out,
                                      conv->slot_stream[slot_of[i]], slot_of[i], nullptr, STAGE_FRONT,
                                      conv->pframes[i].get());
    }
    for (int k = 0; k < nslots; k++) {
        GLS_CUDA(cudaEventRecord(conv->join_ev[k], conv->slot_stream[k]));
        GLS_CUDA(cudaStreamWaitEvent(s, conv->join_ev[k], 0));
    }
    GLS_TRY(result);
    // the work list: rebuilt when the batch changes (never while capturing:
    // a recording runs right after an identical run)
    std::vector<uint64_t> key = batch_key(frames, n, flags);
    if (key.empty() || key != conv->plan_key) {
        if (capturing) return set_error(GLS_ERR_INVALID_ARG, "persistent batch plan changed during capture");
        GLS_TRY(persistent_plan(conv, frames, n));
        conv->plan_key = key;
        conv->plan_grid = persistent_grid(conv->device);
        if (conv->plan_grid <= 0) return set_error(GLS_ERR_CUDA, "persistent kernel occupancy query failed");
    }
    GLS_CUDA(cudaMemsetAsync(conv->plan_cnt.p, 0, size_t(conv->plan_levels) * sizeof(PCounters), s));
    GLS_CUDA(cudaMemsetAsync(conv->plan_ctl.p, 0, 2 * sizeof(int), s));
    {
        KScope k(conv->prof, KC_PERSISTENT, s);
        int* ctl = static_cast<int*>(conv->plan_ctl.p);
        launch_pyramid_persistent(static_cast<const PTask*>(conv->plan_task_buf.p), conv->plan_tasks,
                                  static_cast<const PLevel*>(conv->plan_level_buf.p),
                                  static_cast<PCounters*>(conv->plan_cnt.p), ctl, ctl + 1, kPersistentWaitNs,
                                  conv->plan_grid, s);
    }
    GLS_CUDA(cudaGetLastError());
    // outputs on the slot streams again
    GLS_CUDA(cudaEventRecord(conv->fork_ev, s));
    for (int k = 0; k < nslots; k++) GLS_CUDA(cudaStreamWaitEvent(conv->slot_stream[k], conv->fork_ev, 0));
    for (int oi = 0; oi < n && result == GLS_OK; oi++) {
        const int i = order[oi];
        gls_frame_desc& f = frames[i];
        result = demosaic_run<__half>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params, flags, &f.out,
                                      conv->slot_stream[slot_of[i]], slot_of[i], nullptr, STAGE_OUTPUT,
                                      conv->pframes[i].get());
    }
    for (int k = 0; k < nslots; k++) {
        GLS_CUDA(cudaEventRecord(conv->join_ev[k], conv->slot_stream[k]));
        GLS_CUDA(cudaStreamWaitEvent(s, conv->join_ev[k], 0));
    }
    return result;
}

// The persistent kernel's error word after its batch (synchronises s).
static gls_status persistent_status(gls_converter* conv, cudaStream_t s) {
    int ctl[2] = {0, 0};
    GLS_CUDA(cudaMemcpyAsync(ctl, conv->plan_ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost, s));
    GLS_CUDA(cudaStreamSynchronize(s));
    if (ctl[1]) {
        static const char* const kTypes[4] = {"reconstruct", "covariance", "eigen-solve", "block-matching"};
        return set_error(GLS_ERR_TIMEOUT, "persistent batch: a %s task waited past the limit for its inputs",
                         kTypes[(ctl[1] - 1) & 3]);
    }
    return GLS_OK;
}

// Frames to slot streams, largest first onto the least-loaded slot (the
// longest-processing-time rule), then the fork / per-slot runs / join on s.
static gls_status enqueue_batch(gls_converter* conv, gls_frame_desc* frames, int n, uint32_t flags, cudaStream_t s,
                                bool capturing = false) {
    const int nslots = n < kSlots ? n : kSlots;
    std::vector<int> order(n), slot_of(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return size_t(frames[a].width) * frames[a].height > size_t(frames[b].width) * frames[b].height;
    });
    std::vector<size_t> load(nslots, 0);
    for (int i : order) {
        int k = 0;
        for (int j = 1; j < nslots; j++)
            if (load[j] < load[k]) k = j;
        slot_of[i] = k;
        load[k] += size_t(frames[i].width) * frames[i].height;
    }
    if (flags & GLS_PERSISTENT) return persistent_batch(conv, frames, n, flags, s, order, slot_of, nslots, capturing);
    const bool host_io = flags & GLS_HOST_IO;
    std::vector<SlotCopies> cps(nslots);
    GLS_CUDA(cudaEventRecord(conv->fork_ev, s));
    for (int k = 0; k < nslots; k++) {
        GLS_CUDA(cudaStreamWaitEvent(conv->slot_stream[k], conv->fork_ev, 0));
        cps[k] = {conv->cin_stream[k], conv->cout_stream[k], conv->raw_free[k], conv->raw_ready[k],
                  conv->out_ready[k], conv->out_free[k]};
        if (host_io) {  // both staging buffers start free, after the caller's work
            GLS_CUDA(cudaEventRecord(conv->raw_free[k], conv->slot_stream[k]));
            GLS_CUDA(cudaEventRecord(conv->out_free[k], conv->slot_stream[k]));
        }
    }
    gls_status result = GLS_OK;
    for (int oi = 0; oi < n && result == GLS_OK; oi++) {
        const int i = order[oi];
        gls_frame_desc& f = frames[i];
        const int k = slot_of[i];
        const SlotCopies* cp = host_io ? &cps[k] : nullptr;
        result = (flags & GLS_FP16_STORAGE)
                     ? demosaic_run<__half>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params, flags,
                                            &f.out, conv->slot_stream[k], k, cp)
                     : demosaic_run<float>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params, flags,
                                           &f.out, conv->slot_stream[k], k, cp);
    }
    // join (also on error, so the caller's stream orders after whatever was
    // queued), downloads included
    for (int k = 0; k < nslots; k++) {
        if (host_io) GLS_CUDA(cudaStreamWaitEvent(conv->slot_stream[k], conv->out_free[k], 0));
        GLS_CUDA(cudaEventRecord(conv->join_ev[k], conv->slot_stream[k]));
        GLS_CUDA(cudaStreamWaitEvent(s, conv->join_ev[k], 0));
    }
    return result;
}

}  // namespace gls

extern "C" {

const char* gls_last_error_message(void) { return g_last_error.c_str(); }

const char* gls_version(void) {
    return "glscam 0.1 (sm_100a; demosaic, pyramid PCA block-matching denoise)";
}

gls_status gls_persistent_selftest(int32_t device, int64_t limit_ns, int32_t* err_word) {
    clear_error();
    if (limit_ns <= 0 || limit_ns > 10000000000ll) return set_error(GLS_ERR_INVALID_ARG, "limit_ns out of range");
    GLS_CUDA(cudaSetDevice(device));
    // one eigen-solve task of a level that lists one covariance row but
    // no covariance task: its count never arrives
    PLevel lv{};
    lv.n_cov = 1;
    lv.coarser = -1;
    const PTask task{0u, uint32_t(PT_EIG) << 30};
    DevBuf b_lv, b_task, b_cnt, b_ctl;
    gls_status st = b_lv.ensure(sizeof(PLevel));
    if (st == GLS_OK) st = b_task.ensure(sizeof(PTask));
    if (st == GLS_OK) st = b_cnt.ensure(sizeof(PCounters));
    if (st == GLS_OK) st = b_ctl.ensure(2 * sizeof(int));
    int ctl[2] = {0, 0};
    cudaError_t e = cudaSuccess;
    if (st == GLS_OK) {
        e = cudaMemcpy(b_lv.p, &lv, sizeof(lv), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b_task.p, &task, sizeof(task), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(b_cnt.p, 0, sizeof(PCounters));
        if (e == cudaSuccess) e = cudaMemset(b_ctl.p, 0, 2 * sizeof(int));
        if (e == cudaSuccess) {
            int* c = static_cast<int*>(b_ctl.p);
            launch_pyramid_persistent(static_cast<const PTask*>(b_task.p), 1, static_cast<const PLevel*>(b_lv.p),
                                      static_cast<PCounters*>(b_cnt.p), c, c + 1, limit_ns, 1, nullptr);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(ctl, b_ctl.p, sizeof(ctl), cudaMemcpyDeviceToHost);
    }
    for (DevBuf* b : {&b_lv, &b_task, &b_cnt, &b_ctl}) b->release();
    if (st != GLS_OK) return st;
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "persistent self-test: %s", cudaGetErrorString(e));
    if (err_word) *err_word = ctl[1];
    if (ctl[1]) return set_error(GLS_ERR_TIMEOUT, "persistent self-test: the wait ran out (error word %d)", ctl[1]);
    return GLS_OK;
}

gls_status gls_device_memory(uint64_t* current_bytes, uint64_t* peak_bytes, int32_t reset_peak) {
    clear_error();
    const long long now = g_dev_bytes.load();
    if (current_bytes) *current_bytes = uint64_t(now);
    if (peak_bytes) *peak_bytes = uint64_t(g_dev_peak.load());
    if (reset_peak) g_dev_peak.store(now);
    return GLS_OK;
}

gls_status gls_converter_create(int32_t device, const uint8_t* icc, size_t icc_len, int32_t calibrate_from_image,
                                gls_converter** out) {
    clear_error();
    if (!out) return set_error(GLS_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    if (icc && icc_len)
        return set_error(GLS_ERR_UNSUPPORTED, "ICC profiles are not part of this path; pass xyz_rgb in the parameters");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n)
        return set_error(GLS_ERR_CUDA, "no CUDA device %d (%s)", device, e != cudaSuccess ? cudaGetErrorString(e) : "out of range");
    gls_converter* c = new (std::nothrow) gls_converter();
    if (!c) return set_error(GLS_ERR_OOM, "host allocation failed");
    c->device = device;
    c->calibrate = calibrate_from_image != 0;
    *out = c;
    return GLS_OK;
}

gls_status gls_converter_destroy(gls_converter* conv) {
    clear_error();
    if (!conv) return GLS_OK;
    cudaSetDevice(conv->device);
    cudaDeviceSynchronize();
    for (int k = 0; k < kSlots; k++) {
        conv->p32s[k].release();
        conv->p16s[k].release();
        for (cudaStream_t st : {conv->slot_stream[k], conv->cin_stream[k], conv->cout_stream[k]})
            if (st) cudaStreamDestroy(st);
        for (cudaEvent_t e : {conv->join_ev[k], conv->raw_free[k], conv->raw_ready[k], conv->out_ready[k],
                              conv->out_free[k]})
            if (e) cudaEventDestroy(e);
    }
    if (conv->fork_ev) cudaEventDestroy(conv->fork_ev);
    if (conv->graph_exec) cudaGraphExecDestroy(conv->graph_exec);
    for (auto& pf : conv->pframes) pf->release();
    for (DevBuf* b : {&conv->plan_task_buf, &conv->plan_level_buf, &conv->plan_cnt, &conv->plan_ctl}) b->release();
    for (DevBuf* b : {&conv->adj_gden[0], &conv->adj_gden[1], &conv->adj_rec, &conv->adj_glayer, &conv->adj_gpca,
                      &conv->adj_gup, &conv->adj_part, &conv->adj_loss, &conv->adj_target, &conv->adj_gimg,
                      &conv->adj_gp1, &conv->adj_jvp, &conv->adj_jvp_part, &conv->adj_gout, &conv->nlf_scratch,
                      &conv->nlf_mean, &conv->nlf_var, &conv->nlf_stats})
        b->release();
    delete conv;
    return GLS_OK;
}

gls_status gls_demosaic(gls_converter* conv, const uint16_t* raw, int32_t width, int32_t height,
                        size_t raw_stride_bytes, const gls_demosaic_params* params, uint32_t flags,
                        gls_image_view* out, void* stream) {
    clear_error();
    if (!conv || !raw || !out) return set_error(GLS_ERR_INVALID_ARG, "converter, raw and out must not be NULL");
    GLS_TRY(check_params(params, width, height));
    GLS_TRY(check_post(params, flags));
    if (raw_stride_bytes == 0) raw_stride_bytes = size_t(width) * 2;
    if (raw_stride_bytes < size_t(width) * 2) return set_error(GLS_ERR_INVALID_ARG, "raw stride too small");
    if (out->dtype != GLS_F32 && out->dtype != GLS_F16) return set_error(GLS_ERR_INVALID_ARG, "output dtype must be F32 or F16");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (flags & GLS_FP16_STORAGE)
        return demosaic_run<__half>(conv, raw, width, height, raw_stride_bytes, params, flags, out, s);
    return demosaic_run<float>(conv, raw, width, height, raw_stride_bytes, params, flags, out, s);
}

gls_status gls_demosaic_batch(gls_converter* conv, gls_frame_desc* frames, int32_t n_frames, uint32_t flags,
                              void* stream) {
    clear_error();
    if (!conv || (!frames && n_frames > 0) || n_frames < 0) return set_error(GLS_ERR_INVALID_ARG, "bad batch");
    for (int i = 0; i < n_frames; i++) {  // validate every frame before any work is queued
        gls_frame_desc& f = frames[i];
        GLS_TRY(check_post(f.params, flags));
        if (!f.raw) return set_error(GLS_ERR_INVALID_ARG, "frame %d: raw is NULL", i);
        gls_status st = check_params(f.params, f.width, f.height);
        if (st != GLS_OK) return st;
        if (f.raw_stride_bytes == 0) f.raw_stride_bytes = size_t(f.width) * 2;
        if (f.raw_stride_bytes < size_t(f.width) * 2) return set_error(GLS_ERR_INVALID_ARG, "frame %d: raw stride", i);
        if (f.out.dtype != GLS_F32 && f.out.dtype != GLS_F16)
            return set_error(GLS_ERR_INVALID_ARG, "frame %d: output dtype must be F32 or F16", i);
    }
    const bool persistent = flags & GLS_PERSISTENT;
    if (persistent) {
        if (!(flags & GLS_FP16_STORAGE) || !(flags & GLS_DENOISE))
            return set_error(GLS_ERR_INVALID_ARG, "GLS_PERSISTENT runs the FP16-storage path with noise reduction");
        if (flags & (GLS_HOST_IO | GLS_POSTPROCESS | GLS_HOST_PCA))
            return set_error(GLS_ERR_UNSUPPORTED, "GLS_PERSISTENT takes device buffers, without post-processing "
                                                  "or host PCA");
        if (conv->calibrate) return set_error(GLS_ERR_UNSUPPORTED, "GLS_PERSISTENT cannot run a calibrating converter");
        for (int i = 0; i < n_frames; i++)
            if (!frames[i].out.data)
                return set_error(GLS_ERR_INVALID_ARG, "GLS_PERSISTENT needs caller-owned outputs (frame %d)", i);
    }
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!persistent && ((flags & GLS_HOST_PCA) || n_frames == 1)) {
        // per-level host synchronisation serialises anyway: one frame after the other
        for (int i = 0; i < n_frames; i++) {
            gls_frame_desc& f = frames[i];
            gls_status st = (flags & GLS_FP16_STORAGE)
                                ? demosaic_run<__half>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params,
                                                       flags & ~GLS_SYNC, &f.out, s)
                                : demosaic_run<float>(conv, f.raw, f.width, f.height, f.raw_stride_bytes, f.params,
                                                      flags & ~GLS_SYNC, &f.out, s);
            if (st != GLS_OK) return st;
        }
        if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(s));
        return GLS_OK;
    }
    if (!conv->fork_ev) {
        GLS_CUDA(cudaEventCreateWithFlags(&conv->fork_ev, cudaEventDisableTiming));
        // slot k one priority step below slot k - 1: the slots' frames finish
        // one after another, lower slots filling the gaps, so each frame's
        // copy-out overlaps the later frames' work instead of all of them
        // queueing at the end of the batch
        int least = 0, greatest = 0;
        GLS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        for (int k = 0; k < kSlots; k++) {
            const int prio = std::min(least, greatest + k);
            GLS_CUDA(cudaStreamCreateWithPriority(&conv->slot_stream[k], cudaStreamNonBlocking, prio));
            GLS_CUDA(cudaStreamCreateWithFlags(&conv->cin_stream[k], cudaStreamNonBlocking));
            GLS_CUDA(cudaStreamCreateWithFlags(&conv->cout_stream[k], cudaStreamNonBlocking));
            for (cudaEvent_t* e : {&conv->join_ev[k], &conv->raw_free[k], &conv->raw_ready[k], &conv->out_ready[k],
                                   &conv->out_free[k]})
                GLS_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        }
    }
    const bool graph = flags & GLS_GRAPH;
    std::vector<uint64_t> key;
    if (graph) {
        if (flags & GLS_HOST_PCA) return set_error(GLS_ERR_INVALID_ARG, "GLS_GRAPH needs the device PCA");
        if (!s) return set_error(GLS_ERR_INVALID_ARG, "GLS_GRAPH needs a stream other than the legacy default stream");
        if (conv->prof.on) return set_error(GLS_ERR_INVALID_ARG, "GLS_GRAPH cannot run with profiling enabled");
        if (conv->calibrate)
            return set_error(GLS_ERR_INVALID_ARG, "GLS_GRAPH cannot record a calibrating converter's host reads");
        key = batch_key(frames, n_frames, flags);
        if (!key.empty() && conv->graph_exec && key == conv->graph_key) {  // replay
            GLS_CUDA(cudaGraphLaunch(conv->graph_exec, s));
            if (conv->graph_persistent) return persistent_status(conv, s);
            if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(s));
            return GLS_OK;
        }
        if (key.empty()) return set_error(GLS_ERR_INVALID_ARG, "GLS_GRAPH needs caller-owned outputs");
    }
    gls_status result = enqueue_batch(conv, frames, n_frames, flags & ~(GLS_SYNC | GLS_GRAPH), s);
    if (result == GLS_OK && persistent) result = persistent_status(conv, s);
    if (result == GLS_OK && graph) {
        // record the same launch sequence (allocations and one-time set-up
        // are done by the run above) for replays of this batch
        GLS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        const gls_status cap = enqueue_batch(conv, frames, n_frames, flags & ~(GLS_SYNC | GLS_GRAPH), s, true);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if (cap != GLS_OK) {
            if (g) cudaGraphDestroy(g);
            return cap;
        }
        if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e));
        if (conv->graph_exec) cudaGraphExecDestroy(conv->graph_exec);
        conv->graph_exec = nullptr;
        // kernel nodes keep the slot streams' priorities (captured per node)
        const cudaError_t ie = cudaGraphInstantiateWithFlags(&conv->graph_exec, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            conv->graph_exec = nullptr;
            return set_error(GLS_ERR_CUDA, "batch graph instantiation: %s", cudaGetErrorString(ie));
        }
        conv->graph_key = key;
        conv->graph_persistent = persistent;
    }
    if (result != GLS_OK) return result;
    if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(s));
    return GLS_OK;
}

gls_status gls_pyramid_denoise(gls_converter* conv, const gls_image_view* ycc, const gls_image_view* gradient,
                               const gls_demosaic_params* params, uint32_t flags, gls_image_view* out, void* stream) {
    clear_error();
    if (!conv || !ycc || !gradient || !out || !ycc->data || !gradient->data)
        return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (!params) return set_error(GLS_ERR_INVALID_ARG, "params is NULL");
    if (params->levels < 1 || params->levels > GLS_MAX_LEVELS) return set_error(GLS_ERR_INVALID_ARG, "levels must be 1..5");
    if (gradient->width != ycc->width || gradient->height != ycc->height)
        return set_error(GLS_ERR_INVALID_ARG, "gradient and image sizes differ");
    if (ycc->width < 1 || ycc->height < 1 || (ycc->width >> (params->levels - 1)) < 1 ||
        (ycc->height >> (params->levels - 1)) < 1)
        return set_error(GLS_ERR_INVALID_ARG, "image too small for the pyramid");
    if (out->dtype != GLS_F32 && out->dtype != GLS_F16) return set_error(GLS_ERR_INVALID_ARG, "output dtype must be F32 or F16");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (flags & GLS_FP16_STORAGE) return pyramid_only<__half>(conv, ycc, gradient, params, flags, out, s);
    return pyramid_only<float>(conv, ycc, gradient, params, flags, out, s);
}

gls_status gls_converter_plane(gls_converter* conv, int32_t which, gls_image_view* view) {
    clear_error();
    if (!conv || !view) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (which == GLS_PLANE_NLF_MEAN || which == GLS_PLANE_NLF_VAR) {
        if (!conv->nlf_mw) return set_error(GLS_ERR_INVALID_ARG, "no raw noise measurement has run");
        *view = {which == GLS_PLANE_NLF_MEAN ? conv->nlf_mean.p : conv->nlf_var.p, conv->nlf_mw, conv->nlf_mh, 4,
                 GLS_F32, size_t(conv->nlf_mw) * 4 * sizeof(float)};
        return GLS_OK;
    }
    if (which == GLS_PLANE_NLF_STATS) {
        if (!conv->nlf_sw) return set_error(GLS_ERR_INVALID_ARG, "no YCbCr noise measurement has run");
        *view = {conv->nlf_stats.p, conv->nlf_sw, conv->nlf_sh, 4, GLS_F32, size_t(conv->nlf_sw) * 4 * sizeof(float)};
        return GLS_OK;
    }
    if (conv->last_storage < 0) return set_error(GLS_ERR_INVALID_ARG, "no frame has been processed");
    const bool h = conv->last_storage == GLS_F16;
    const int w = conv->last_w, hh = conv->last_h;
    const size_t es = h ? 2 : 4;
    auto pick = [&](DevBuf& b16, DevBuf& b32) { return h ? b16.p : b32.p; };
    view->dtype = h ? GLS_F16 : GLS_F32;
    switch (which) {
        case GLS_PLANE_SCALED_RAW:
            *view = {pick(conv->p16.scaled, conv->p32.scaled), w, hh, 1, view->dtype, size_t(w) * es};
            return GLS_OK;
        case GLS_PLANE_GRADIENT:
            *view = {pick(conv->p16.grad, conv->p32.grad), w, hh, 2, view->dtype, size_t(w) * 2 * es};
            return GLS_OK;
        case GLS_PLANE_DEMOSAIC:
        case GLS_PLANE_OUTPUT:
            if (which == GLS_PLANE_DEMOSAIC || !conv->last_denoise) {
                *view = {pick(conv->p16.A, conv->p32.A), w, hh, 4, view->dtype, size_t(w) * 4 * es};
                return GLS_OK;
            }
            return set_error(GLS_ERR_INVALID_ARG, "the denoised output lives in the caller's view");
        case GLS_PLANE_DESPECKLED:
            *view = {pick(conv->p16.B, conv->p32.B), w, hh, 4, view->dtype, size_t(w) * 4 * es};
            return GLS_OK;
        case GLS_PLANE_ADJ_DESPECKLED:
            if (!conv->adj_gimg_w) return set_error(GLS_ERR_INVALID_ARG, "no gls_demosaic_denoise_vjp has run");
            *view = {conv->adj_gimg.p, conv->adj_gimg_w, conv->adj_gimg_h, 3, GLS_F32,
                     size_t(conv->adj_gimg_w) * 3 * sizeof(float)};
            return GLS_OK;
        default:
            if (which >= GLS_PLANE_DENOISED_L0 && which < GLS_PLANE_DENOISED_L0 + conv->last_levels) {
                const int l = which - GLS_PLANE_DENOISED_L0;
                *view = {pick(conv->p16.den[l], conv->p32.den[l]), w >> l, hh >> l, 4, view->dtype,
                         size_t(w >> l) * 4 * es};
                return GLS_OK;
            }
            return set_error(GLS_ERR_INVALID_ARG, "unknown plane %d", which);
    }
}

gls_status gls_converter_pca_basis(gls_converter* conv, int32_t level, float* basis25x8) {
    clear_error();
    if (!conv || !basis25x8) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (conv->last_storage < 0 || level < 0 || level >= conv->last_levels)
        return set_error(GLS_ERR_INVALID_ARG, "no PCA basis for level %d", level);
    GLS_CUDA(cudaSetDevice(conv->device));
    const float* b = static_cast<const float*>(conv->last_storage == GLS_F16 ? conv->p16.basis.p : conv->p32.basis.p);
    GLS_CUDA(cudaDeviceSynchronize());
    GLS_CUDA(cudaMemcpy(basis25x8, b + level * 200, sizeof(float) * 200, cudaMemcpyDeviceToHost));
    return GLS_OK;
}

gls_status gls_copy_view(const gls_image_view* src, gls_image_view* dst, int32_t direction, void* stream) {
    clear_error();
    if (!src || !dst || !src->data || !dst->data) return set_error(GLS_ERR_INVALID_ARG, "NULL view");
    if (src->width != dst->width || src->height != dst->height || src->channels != dst->channels ||
        src->dtype != dst->dtype)
        return set_error(GLS_ERR_INVALID_ARG, "views differ in shape or dtype");
    const size_t es = src->dtype == GLS_F32 ? 4 : 2;
    const size_t row = size_t(src->width) * src->channels * es;
    if (src->stride_bytes < row || dst->stride_bytes < row) return set_error(GLS_ERR_INVALID_ARG, "stride too small");
    cudaMemcpyKind kind = direction == GLS_COPY_D2H   ? cudaMemcpyDeviceToHost
                          : direction == GLS_COPY_D2D ? cudaMemcpyDeviceToDevice
                                                      : cudaMemcpyHostToDevice;
    if (direction < 0 || direction > 2) return set_error(GLS_ERR_INVALID_ARG, "bad direction");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    GLS_CUDA(cudaMemcpy2DAsync(dst->data, dst->stride_bytes, src->data, src->stride_bytes, row, src->height, kind, s));
    if (direction == GLS_COPY_D2H) GLS_CUDA(cudaStreamSynchronize(s));
    return GLS_OK;
}

gls_status gls_converter_set_profiling(gls_converter* conv, int32_t enable) {
    clear_error();
    if (!conv) return set_error(GLS_ERR_INVALID_ARG, "NULL converter");
    GLS_CUDA(cudaSetDevice(conv->device));
    if (conv->prof.on && !enable) {
        GLS_CUDA(cudaDeviceSynchronize());
        conv->prof.drain();
    }
    conv->prof.on = enable != 0;
    return GLS_OK;
}

gls_status gls_converter_stats(gls_converter* conv, gls_kernel_stat* stats, int32_t max_stats, int32_t* n_stats) {
    clear_error();
    if (!conv || !n_stats) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    GLS_CUDA(cudaSetDevice(conv->device));
    GLS_CUDA(cudaDeviceSynchronize());
    conv->prof.drain();
    *n_stats = KC_COUNT;
    for (int i = 0; i < KC_COUNT && i < max_stats && stats; i++)
        stats[i] = {kKcNames[i], conv->prof.launches[i], conv->prof.ms[i]};
    return GLS_OK;
}

gls_status gls_converter_reset_stats(gls_converter* conv) {
    clear_error();
    if (!conv) return set_error(GLS_ERR_INVALID_ARG, "NULL converter");
    GLS_CUDA(cudaSetDevice(conv->device));
    GLS_CUDA(cudaDeviceSynchronize());
    conv->prof.drain();
    for (int i = 0; i < KC_COUNT; i++) {
        conv->prof.launches[i] = 0;
        conv->prof.ms[i] = 0;
    }
    return GLS_OK;
}

gls_status gls_calibration_fill(int32_t camera, int32_t iso, gls_demosaic_params* params) {
    clear_error();
    return calibration_fill(camera, iso, params);
}

gls_status gls_gaussian_bilinear_taps(float radius, float* taps, int32_t max_taps, int32_t* n_taps) {
    clear_error();
    if (!taps || !n_taps || !(radius > 0.f) || radius > 30.f) return set_error(GLS_ERR_INVALID_ARG, "bad arguments");
    const int n = gaussian_taps(radius, taps, max_taps);
    *n_taps = n < 0 ? -n : n;
    if (n < 0) return set_error(GLS_ERR_INVALID_ARG, "max_taps too small (%d needed)", -n);
    return GLS_OK;
}


gls_status gls_demosaic_denoise_vjp(gls_converter* conv, const uint16_t* raw, int32_t width, int32_t height,
                                    size_t raw_stride_bytes, const gls_demosaic_params* params,
                                    const gls_image_view* target, uint32_t flags, double* loss, float* grad,
                                    void* stream) {
    clear_error();
    if (!conv || !raw || !params || !target || !target->data || !grad)
        return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (params->levels < 1 || params->levels > GLS_MAX_LEVELS) return set_error(GLS_ERR_INVALID_ARG, "bad levels");
    if (target->width != width || target->height != height || target->dtype != GLS_F32 ||
        (target->channels != 3 && target->channels != 4))
        return set_error(GLS_ERR_INVALID_ARG, "target must be a %dx%d GLS_F32 RGB or RGBA view", width, height);
    const size_t trow = size_t(width) * target->channels * 4;
    const size_t tstride_b = target->stride_bytes ? target->stride_bytes : trow;
    if (tstride_b < trow || tstride_b % 4) return set_error(GLS_ERR_INVALID_ARG, "bad target stride");
    if (conv->calibrate)
        return set_error(GLS_ERR_UNSUPPORTED, "the gradient is taken with respect to the given noise models; "
                                              "a calibrating converter replaces them with measured ones");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    gls_image_view out{};  // converter-owned FP32 output
    out.dtype = GLS_F32;
    const uint32_t fw = GLS_DENOISE | (flags & GLS_HOST_IO);
    conv->keep_nc = true;
    const gls_status fst = demosaic_run<float>(conv, raw, width, height, raw_stride_bytes, params, fw, &out, s);
    conv->keep_nc = false;
    GLS_TRY(fst);
    const float* tp = static_cast<const float*>(target->data);
    if ((flags & GLS_HOST_IO) || tstride_b != trow) {
        GLS_TRY(conv->adj_target.ensure(size_t(height) * trow));
        GLS_CUDA(cudaMemcpy2DAsync(conv->adj_target.p, trow, target->data, tstride_b, trow, height,
                                   (flags & GLS_HOST_IO) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
        tp = static_cast<const float*>(conv->adj_target.p);
    }
    return adjoint_run(conv, params, tp, target->channels, nullptr, true, loss, grad, s);
}

gls_status gls_pyramid_denoise_vjp(gls_converter* conv, const gls_image_view* ycc, const gls_image_view* gradient,
                                   const gls_demosaic_params* params, const gls_image_view* g_out, uint32_t flags,
                                   float* grad, gls_image_view* g_ycc, void* stream) {
    clear_error();
    if (!conv || !ycc || !gradient || !params || !g_out || !g_out->data || !grad)
        return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (params->levels < 1 || params->levels > GLS_MAX_LEVELS) return set_error(GLS_ERR_INVALID_ARG, "bad levels");
    const int w = ycc->width, h = ycc->height;
    if (gradient->width != w || gradient->height != h) return set_error(GLS_ERR_INVALID_ARG, "gradient and image sizes differ");
    if (w < 1 || h < 1 || (w >> (params->levels - 1)) < 1 || (h >> (params->levels - 1)) < 1)
        return set_error(GLS_ERR_INVALID_ARG, "image too small for the pyramid");
    auto check3 = [&](const gls_image_view* v, const char* what) -> gls_status {
        if (v->width != w || v->height != h || v->dtype != GLS_F32 || (v->channels != 3 && v->channels != 4))
            return set_error(GLS_ERR_INVALID_ARG, "%s must be a %dx%d GLS_F32 view of 3 or 4 channels", what, w, h);
        const size_t row = size_t(w) * v->channels * 4;
        const size_t st = v->stride_bytes ? v->stride_bytes : row;
        if (st < row || st % 4) return set_error(GLS_ERR_INVALID_ARG, "bad %s stride", what);
        return GLS_OK;
    };
    GLS_TRY(check3(g_out, "g_out"));
    if (g_ycc) {
        if (!g_ycc->data) return set_error(GLS_ERR_INVALID_ARG, "g_ycc has no data");
        GLS_TRY(check3(g_ycc, "g_ycc"));
    }
    if (conv->calibrate)
        return set_error(GLS_ERR_UNSUPPORTED, "the gradient is taken with respect to the given noise models; "
                                              "a calibrating converter replaces them with measured ones");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool host_io = flags & GLS_HOST_IO;
    gls_image_view out{};  // converter-owned FP32 output
    out.dtype = GLS_F32;
    conv->keep_nc = true;
    const gls_status fst = pyramid_only<float>(conv, ycc, gradient, params, GLS_DENOISE | (flags & GLS_HOST_IO), &out, s);
    conv->keep_nc = false;
    GLS_TRY(fst);
    const size_t n = size_t(w) * h;
    GLS_TRY(conv->adj_gout.ensure(n * 3 * sizeof(float)));
    float* g3 = static_cast<float*>(conv->adj_gout.p);
    {  // the cotangent into a packed 3-channel plane
        const size_t row = size_t(w) * g_out->channels * 4;
        const size_t st = g_out->stride_bytes ? g_out->stride_bytes : row;
        const float* src = static_cast<const float*>(g_out->data);
        size_t pitch = st / 4;
        if (host_io) {
            GLS_TRY(conv->adj_target.ensure(size_t(h) * row));
            GLS_CUDA(cudaMemcpy2DAsync(conv->adj_target.p, row, g_out->data, st, row, h, cudaMemcpyHostToDevice, s));
            src = static_cast<const float*>(conv->adj_target.p);
            pitch = row / 4;
        }
        launch_pack3(src, pitch, g_out->channels, g3, w, h, s);
    }
    GLS_TRY(adjoint_run(conv, params, nullptr, 0, g3, false, nullptr, grad, s));
    if (g_ycc) {
        const size_t row = size_t(w) * g_ycc->channels * 4;
        const size_t st = g_ycc->stride_bytes ? g_ycc->stride_bytes : row;
        const float* gi = static_cast<const float*>(conv->adj_gimg.p);  // level 0 first
        if (host_io) {
            GLS_TRY(conv->adj_target.ensure(size_t(h) * row));
            launch_unpack3(gi, static_cast<float*>(conv->adj_target.p), row / 4, g_ycc->channels, w, h, s);
            GLS_CUDA(cudaMemcpy2DAsync(g_ycc->data, st, conv->adj_target.p, row, row, h, cudaMemcpyDeviceToHost, s));
        } else {
            launch_unpack3(gi, static_cast<float*>(g_ycc->data), st / 4, g_ycc->channels, w, h, s);
        }
        GLS_CUDA(cudaGetLastError());
    }
    GLS_CUDA(cudaStreamSynchronize(s));
    return GLS_OK;
}


gls_status gls_block_match_tiles(int32_t* entries, int32_t max_entries, int32_t* n) {
    clear_error();
    if (!n || (max_entries > 0 && !entries)) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    std::vector<int> buf(3 * size_t(std::max(max_entries, 0)));
    const int c = bm_tile_list(buf.data(), std::max(max_entries, 0));
    for (int i = 0; i < std::min(c, max_entries) * 3; i++) entries[i] = buf[i];
    *n = c;
    return GLS_OK;
}

gls_status gls_grain_tables(uint32_t seed, int32_t* perm, float* grad) {
    clear_error();
    if (!perm || !grad) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    int pi[kNoiseSize];
    noise_tables(seed, pi, grad);
    for (int i = 0; i < kNoiseSize; i++) perm[i] = pi[i];
    return GLS_OK;
}
}  // extern "C"

// ---- noise-model measurement (calibrateFromImage)

gls_status gls_measure_raw_nlf(gls_converter* conv, const gls_image_view* scaled_raw, int32_t bayer_pattern,
                               float exposure_multiplier, gls_raw_nlf* out, void* stream) {
    clear_error();
    if (!conv || !scaled_raw || !scaled_raw->data || !out) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (bayer_pattern < 0 || bayer_pattern > 3) return set_error(GLS_ERR_INVALID_ARG, "bad Bayer pattern");
    if (scaled_raw->channels != 1) return set_error(GLS_ERR_INVALID_ARG, "the scaled raw view must have 1 channel");
    if (scaled_raw->width < 2 || scaled_raw->height < 2) return set_error(GLS_ERR_INVALID_ARG, "frame too small");
    const size_t es = scaled_raw->dtype == GLS_F32 ? 4 : scaled_raw->dtype == GLS_F16 ? 2 : 0;
    if (!es) return set_error(GLS_ERR_INVALID_ARG, "scaled raw dtype must be F32 or F16");
    if (scaled_raw->stride_bytes % es) return set_error(GLS_ERR_INVALID_ARG, "stride is not a whole number of elements");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (es == 4) {
        Plane<float, 1> pl{static_cast<float*>(scaled_raw->data), scaled_raw->width, scaled_raw->height,
                           scaled_raw->stride_bytes / 4};
        return measure_raw_nlf<float>(conv, pl, bayer_pattern, exposure_multiplier, out, s);
    }
    Plane<__half, 1> pl{static_cast<__half*>(scaled_raw->data), scaled_raw->width, scaled_raw->height,
                        scaled_raw->stride_bytes / 2};
    return measure_raw_nlf<__half>(conv, pl, bayer_pattern, exposure_multiplier, out, s);
}

gls_status gls_measure_ycbcr_nlf(gls_converter* conv, const gls_image_view* ycc, float exposure_multiplier,
                                 gls_ycbcr_nlf* out, void* stream) {
    clear_error();
    if (!conv || !ycc || !ycc->data || !out) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (ycc->channels != 4) return set_error(GLS_ERR_INVALID_ARG, "the YCbCr view must have 4 channels");
    if (ycc->width < 1 || ycc->height < 1) return set_error(GLS_ERR_INVALID_ARG, "empty image");
    const size_t es = ycc->dtype == GLS_F32 ? 4 : ycc->dtype == GLS_F16 ? 2 : 0;
    if (!es) return set_error(GLS_ERR_INVALID_ARG, "YCbCr dtype must be F32 or F16");
    if (ycc->stride_bytes % (4 * es)) return set_error(GLS_ERR_INVALID_ARG, "stride is not a whole number of pixels");
    if (uintptr_t(ycc->data) % (4 * es)) return set_error(GLS_ERR_INVALID_ARG, "YCbCr data must be pixel-aligned");
    GLS_CUDA(cudaSetDevice(conv->device));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (es == 4) {
        Plane<float, 4> pl{static_cast<float*>(ycc->data), ycc->width, ycc->height, ycc->stride_bytes / 4};
        return measure_ycc_nlf<float>(conv, pl, exposure_multiplier, out, s);
    }
    Plane<__half, 4> pl{static_cast<__half*>(ycc->data), ycc->width, ycc->height, ycc->stride_bytes / 2};
    return measure_ycc_nlf<__half>(conv, pl, exposure_multiplier, out, s);
}

gls_status gls_converter_noise_model(gls_converter* conv, gls_raw_nlf* raw, gls_ycbcr_nlf* pyramid,
                                     int32_t max_levels, int32_t* n_levels) {
    clear_error();
    if (!conv) return set_error(GLS_ERR_INVALID_ARG, "NULL converter");
    if (!conv->calibrate) return set_error(GLS_ERR_INVALID_ARG, "the converter was not created to calibrate from images");
    if (!conv->nlf_mw) return set_error(GLS_ERR_INVALID_ARG, "no frame has been measured");
    if (raw) *raw = conv->nlf_raw;
    if (pyramid)
        for (int i = 0; i < conv->nlf_levels && i < max_levels; i++) pyramid[i] = conv->nlf_pyr[i];
    if (n_levels) *n_levels = conv->nlf_levels;
    return GLS_OK;
}
