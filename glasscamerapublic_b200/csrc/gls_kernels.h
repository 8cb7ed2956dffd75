// gls_kernels.h — kernel argument blocks and host launchers of the raw path.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "gls_common.cuh"

struct gls_demosaic_params;
struct gls_raw_nlf;

namespace gls {

// Raise `func`'s dynamic shared-memory limit to `bytes` on the current
// device. The attribute belongs to the device's context, so it is set once
// per (kernel, device) pair; the record of pairs done is guarded by a
// mutex, so converters on several host threads and devices may launch
// concurrently. Returns the CUDA error of the first, failed setting.
cudaError_t ensure_dynamic_smem(const void* func, int bytes);

constexpr int kMaxTaps = 32;

struct ScaleArgs {
    int pattern;
    int black;       // integer black level (DN)
    float k[4];      // scale_mul[c] * 0.9 / 65535, per Bayer channel
    float lsc;       // lens shading strength (0 = off)
    float cx, cy, clen;
};

struct BlurArgs {
    int n1, n2;                  // narrow / wide tap counts (wide taps follow the narrow ones)
    float w[kMaxTaps];           // tap weights
    int ix[kMaxTaps], iy[kMaxTaps];    // floor of the tap offsets
    float fx[kMaxTaps], fy[kMaxTaps];  // fractional parts
    float var0, var1;            // green raw variance (a, b)
    float inv_sqrt45;
};

struct RawDenoiseArgs {
    int pattern;
    float var[4];     // raw NLF b coefficients per channel (R, G, B, G2)
    float strength;   // cross-denoise strength
    int fast;         // fast exp (FP16-storage path)
};

struct DemosaicArgs {
    int pattern;
    float rv0, rv1, gv0, gv1, bv0, bv1;  // raw variance (a, b) of R, G, B
    int transform;                       // apply m (cam -> YCbCr) to the output
    float m[9];
};

struct Mat3Args {
    float m[9];
};

template <class S>
void launch_scale_raw(const uint16_t* raw, size_t raw_pitch, Plane<S, 1> out, const ScaleArgs& a, cudaStream_t s);
template <class S>
void launch_sobel_blur(Plane<S, 1> raw, Plane<S, 2> out, const BlurArgs& a, cudaStream_t s);
template <class S>
void launch_raw_denoise(Plane<S, 1> bayer, Plane<S, 2> grad, Plane<S, 4> quad, const RawDenoiseArgs& a,
                        cudaStream_t s);
template <class S>
void launch_demosaic(Plane<S, 1> raw, Plane<S, 2> grad, Plane<S, 4> out, const DemosaicArgs& a, cudaStream_t s);
template <class S>
void launch_despeckle(Plane<S, 4> in, Plane<S, 4> out, float va, float vb, cudaStream_t s);
template <class S, class O>
void launch_transform(Plane<S, 4> in, Plane<O, 4> out, const Mat3Args& m, cudaStream_t s);
template <class S, class O>
void launch_convert4(Plane<S, 4> in, Plane<O, 4> out, cudaStream_t s);

// ---- pyramid ----
struct BlockMatchArgs {
    float var_a[3], var_b[3];     // YCbCr NLF of the level
    float tm[3];                  // threshold multipliers (luma, chroma, chroma)
    float chroma_boost, gradient_boost, gradient_threshold;
    float lsc;                    // lens shading correction (0 = off)
    float* nc_out = nullptr;      // FP32 path: the chroma kernel norm per pixel, kept for the adjoint
    bool tensor = false;          // FP16 path: the tensor-core matcher (GLS_BM_TENSOR)
};

struct SubtractArgs {
    float luma_weight, sharpening, nlf_a, nlf_b;
};

// PCA accumulators of one level: the upper triangle of sum p p^T over the
// patches (325, row-major) followed by sum p (25), FP64.
constexpr int kPcaAcc = 25 + 325;
constexpr int kPcaDim = 25, kPcaComp = 8;
// 64-patch chunks per covariance partial row of a level with `chunks`
// chunks: about 372 rows per level (a few per SM) for the fine levels, one
// chunk per row for the coarse ones (short per-block chains), at most 16
__host__ __device__ inline int pca_cov_group(int chunks) {
    const int g = chunks / 372;
    return g < 1 ? 1 : (g > 16 ? 16 : g);
}
int pca_cov_chunks(int w, int h);  // 64-patch chunks of a level
int pca_cov_rows(int w, int h);    // partial rows of a level: chunks / pca_cov_group(chunks), rounded up

template <class S, int C>
void launch_downsample(Plane<S, C> in, Plane<S, C> out, cudaStream_t s);
// a level's image and gradient in one launch (equal sizes)
template <class S>
void launch_downsample_pair(Plane<S, 4> img, Plane<S, 4> img_out, Plane<S, 2> grad, Plane<S, 2> grad_out,
                            cudaStream_t s);
template <class S>
void launch_subtract_noise(Plane<S, 4> in, Plane<S, 4> coarse, Plane<S, 4> coarse_den, Plane<S, 2> grad,
                           Plane<S, 4> out, const SubtractArgs& a, cudaStream_t s);
template <class S>
void launch_pca_cov(Plane<S, 4> img, double* part, cudaStream_t s);
// one block and partial row per 64-patch chunk: `rows` = ceil(patches / 64)
template <class S>
void launch_pca_cov_rows(Plane<S, 4> img, double* part, int rows, cudaStream_t s);
constexpr int kPcaChunk = 64;
void launch_pca_eigen(const double* part, int n_blocks, int n_patches, float* basis /*25x8*/, int* status,
                      cudaStream_t s);
template <class S>
void launch_pca_project(Plane<S, 4> img, const float* basis, Plane<S, 8> out, cudaStream_t s);
// FP32 path: reads the projected `pca` plane; FP16 path: projects on tensor
// cores inside the kernel from `basis` (the pca plane is not used)
template <class S>
void launch_block_match(Plane<S, 4> img, Plane<S, 2> grad, Plane<S, 8> pca, const float* basis, Plane<S, 4> out,
                        const BlockMatchArgs& a, cudaStream_t s);

// the FP16 block matcher's tile-height autotuner decisions: (w, h, height)
// triples of the level sizes seen so far; returns their count
int bm_tile_list(int* whty, int max);

// ---- the persistent batch kernel: every pyramid level of every frame of a
//      batch (reconstruct, covariance, eigen-solve, block matching) in one
//      launch over a device work list, levels ordered by dependency counters
enum PTaskType : uint32_t { PT_SN = 0, PT_COV = 1, PT_EIG = 2, PT_BM = 3 };
struct PTask {
    uint32_t lev;   // index of the (frame, level) descriptor
    uint32_t item;  // type in the top 2 bits; tile / row index below
};
constexpr uint32_t kPTaskItemMask = 0x3fffffffu;
// side of a persistent reconstruct task's tile: 64 x 64 pixels (16 per
// thread), so the per-task fetch and bookkeeping stay small beside the work
constexpr int kPSnTile = 64;
struct PLevel {
    Plane<__half, 4> img, layer, den;  // the level's image, reconstructed layer, denoised output
    Plane<__half, 2> grad;
    Plane<__half, 4> coarse, coarse_den;  // the next coarser level (reconstruct inputs)
    double* part;                         // covariance partial rows
    float* basis;                         // 25 x 8
    int* status;                          // eigen-solve status
    SubtractArgs sa;
    float rx, ry;                         // coarse / fine size ratios
    BlockMatchArgs ba;
    int n_sn, n_cov, n_bm;                // task counts of the level
    int tiles_x;                          // 32-pixel block-matching tiles across the level
    int sn_tiles_x;                       // reconstruct tiles (kPSnTile pixels square) across the level
    int chunks;                           // 64-patch covariance chunks
    int cov_group;                        // chunks per covariance row (pca_cov_group)
    int coarser;                          // descriptor of the next coarser level, -1 at the coarsest
};
struct PCounters {
    int sn, cov, eig, bm;  // tasks of the level finished, per type
};
// blocks the kernel runs as (resident on the device at once)
int persistent_grid(int device);
// tasks[n]; lv, cnt: one per descriptor (cnt zeroed); next: the work
// counter (zeroed); err: 0, or set to 1 + the type of the task whose wait
// ran past limit_ns (the kernel then stops taking tasks)
void launch_pyramid_persistent(const PTask* tasks, int n, const PLevel* lv, PCounters* cnt, int* next, int* err,
                               long long limit_ns, int grid, cudaStream_t s);

// ---- display post-processing (gls_post.cu)
// histogram_data's statistics (demosaic.metal:1360-1369)
struct PostStats {
    float black, white, shadows, highlights, mean, median;
};
template <class S>
struct PostArgs {
    const gls_demosaic_params* params;
    float y2c[9];           // YCbCr -> camera RGB
    bool denoise;           // den[] valid (else rgb is the demosaic output)
    Plane<S, 4> den[5];     // denoised levels, YCbCr
    Plane<S, 4> rgb;        // camera RGB without noise reduction
    Plane<S, 2> grad2;      // level-0 gradient plane
    const uint16_t* raw;    // the raw frame on the device: its first pixel seeds the grain
    uint32_t* hist;         // 256 bins, zero on entry (zeroed when allocated; left zeroed)
    PostStats* stats;
    int* perm;              // kNoiseSize
    float* grad_tab;        // kNoiseSize x 2
    float2* ab;             // post_ab_bytes: the three bands' filtered (a, b)
};
size_t post_ab_bytes(int w, int h);
// returns the number of kernels launched
template <class S, class O>
int launch_post(const PostArgs<S>& pa, Plane<O, 4> out, cudaStream_t s);

// noise-model measurement (gls_nlf.cu): statistics into the given float
// planes (raw: (w/2) x (h/2); YCbCr: the level's size), then the fits, the
// result written to *out (device memory; YCbCr: a[0..2], b[0..2]). scratch:
// nlf_scratch_bytes(). Each returns the number of kernels launched.
size_t nlf_scratch_bytes();
template <class S>
int launch_measure_raw_nlf(Plane<S, 1> scaled, int pattern, Plane<float, 4> mean, Plane<float, 4> var,
                           float exposure, void* scratch, gls_raw_nlf* out, cudaStream_t s);
template <class S>
int launch_measure_ycc_nlf(Plane<S, 4> img, Plane<float, 4> stats, float exposure, void* scratch,
                           gls_raw_nlf* out, cudaStream_t s);

// ---- adjoint of the pyramid (gls_adjoint.cu); FP32 planes, tightly packed
struct AdjointLevelArgs {
    int w, h;
    const float* den;    // 4 ch: the forward's block-matching output (Y, Cb, Cr, luma norm)
    const float* nc;     // 1 ch: the forward's chroma norm
    const float* layer;  // 4 ch: the level's block-matching input
    const float* grad;   // 2 ch
    const float* pca;    // 8 ch, projected with `basis`
    const float* basis;  // 25 x 8 (device)
    const float* g_den;  // 3 ch: dL/d(block-matching output Y, Cb, Cr)
    float* rec;          // 12 per pixel: centre record for the neighbour pass
    float* g_layer;      // 4 ch out: dL/d layer (Y, Cb, Cr)
    float* g_pca;        // 8 ch scratch
    float* part;         // per-block dL/dtheta: luma, chroma, A_Y, B_Y, A_C, B_C
    float var_a[3], var_b[3], tm[3];
    float chroma_boost, gradient_boost, gradient_threshold;
};
struct AdjointHeadArgs {
    float m[9];   // YCbCr -> camera RGB
    float inv_n;  // 1 / (3 pixels)
};
struct AdjointSnArgs {
    int w, h, cw, ch;  // fine and coarse sizes
    float rx, ry;      // coarse / fine
    const float *in, *coarse, *coarse_den, *grad, *g_layer;
    float* g_up;          // 3 ch fine scratch
    float* g_coarse_den;  // 3 ch out at the coarse level
    float* part;          // per-block dL/d nlf_a, dL/d nlf_b
    float luma_weight, sharpening, nlf_a, nlf_b;
    // optional (null: skipped): dL/d of the level's noisy input image, 3 ch
    float* g_in;          // += at the fine level
    float* g_p1;          // 3 ch fine scratch: dL/d(up-sampled coarse noisy image)
    float* g_coarse_img;  // += at the coarse level
};
void launch_adj_head(const float* den0, const float* target, int tstride, int w, int h, const AdjointHeadArgs& a,
                     float* g_den, double* loss_part, cudaStream_t s);
// g_img (3 ch) += the first 3 channels of g_layer (4 ch): the coarsest
// level's block matching reads the level image itself
void launch_add_layer_grad(const float* g_layer, float* g_img, int w, int h, cudaStream_t s);
// g_fine (3 ch, w x h) += transpose of the pyramid down-sampling
// (k_downsample) applied to g_coarse (3 ch, cw x ch)
void launch_down_bwd(const float* g_coarse, int cw, int ch, float* g_fine, int w, int h, cudaStream_t s);

// 3-channel planes (tightly packed) from / to views of 3 or 4 channels
// (pitch in floats; a fourth channel is written as 0)
void launch_pack3(const float* src, size_t pitch_floats, int channels, float* dst, int w, int h, cudaStream_t s);
void launch_unpack3(const float* src, float* dst, size_t pitch_floats, int channels, int w, int h, cudaStream_t s);

// ---- forward-mode tangents of the raw front end (gls_front_jvp.cu)
struct FrontJvpArgs {
    int w, h;
    const float* scaled;   // Bayer plane after the raw branch (forward, FP32)
    const float* scaled0;  // Bayer plane before the raw branch (forward, with high_noise)
    const float* quad;     // despeckled quads of the raw branch (forward)
    const float* grad;    // 2 ch gradient plane (forward)
    int high_noise;       // the raw branch ran
    RawDenoiseArgs raw;
    DemosaicArgs dm;      // transform = cam -> YCbCr
    float despeckle_va, despeckle_vb;
    const float* g_ds;    // 3 ch: dL/d(despeckled YCbCr), from the reverse sweep
    void* scratch;        // front_jvp_scratch_bytes(w, h)
    float* part;          // per block: dL/dtheta30, dL/dtheta31
};
size_t front_jvp_scratch_bytes(int w, int h);
int front_jvp_blocks(int w, int h);
void launch_front_jvp(const FrontJvpArgs& f, cudaStream_t s);
void launch_bm_bwd(const AdjointLevelArgs& a, cudaStream_t s);
void launch_sn_bwd(const AdjointSnArgs& a, cudaStream_t s);
int adjoint_blocks(int w, int h);
int adjoint_sn_blocks(int w, int h);

// host-side eigen-solve of the same accumulators (the reference's per-level
// host PCA, pyramid_processor.cpp:148-149)
void host_pca_basis(const double* part, int n_blocks, int n_patches, float* basis);

// Top-8 basis (row-major 25 x 8, FP32) from eigenpairs sorted by decreasing
// eigenvalue: ev[c] and column c of evec (row stride ld). Columns whose
// eigenvalue is not above 1e-9 x the largest lie in a null space that a
// solver fills arbitrarily (fewer than 26 patches, or a flat level); they
// are completed deterministically by Gram-Schmidt of the unit vectors
// e0, e1, ... against the previous columns. Each column is signed so that
// its largest-magnitude entry (first on ties) is positive. work: 200 doubles.
__host__ __device__ inline void select_pca_basis(const double* ev, const double* evec, int ld, double* work,
                                                 float* basis) {
    const double lam0 = ev[0] > 0.0 ? ev[0] : 0.0;
    const double tol = 1e-9 * lam0;
    int cand = 0;
    bool kept = true;
    for (int c = 0; c < 8; c++) {
        double* v = work + c * 25;
        kept = kept && lam0 > 0.0 && ev[c] > tol;
        if (kept) {
            for (int r = 0; r < 25; r++) v[r] = evec[r * ld + c];
        } else {
            for (int guard = 0; guard < 25; guard++) {
                for (int r = 0; r < 25; r++) v[r] = (r == cand) ? 1.0 : 0.0;
                cand++;
                for (int pass = 0; pass < 2; pass++)
                    for (int k = 0; k < c; k++) {
                        const double* b = work + k * 25;
                        double d = 0;
                        for (int r = 0; r < 25; r++) d += b[r] * v[r];
                        for (int r = 0; r < 25; r++) v[r] -= d * b[r];
                    }
                double nn = 0;
                for (int r = 0; r < 25; r++) nn += v[r] * v[r];
                if (nn > 0.25) {
                    const double inv = 1.0 / sqrt(nn);
                    for (int r = 0; r < 25; r++) v[r] *= inv;
                    break;
                }
            }
        }
        int amax = 0;
        for (int r = 1; r < 25; r++)
            if (fabs(v[r]) > fabs(v[amax])) amax = r;
        const double sgn = v[amax] < 0 ? -1.0 : 1.0;
        for (int r = 0; r < 25; r++) v[r] *= sgn;
    }
    for (int c = 0; c < 8; c++)
        for (int r = 0; r < 25; r++) basis[r * 8 + c] = float(work[c * 25 + r]);
}

}  // namespace gls
