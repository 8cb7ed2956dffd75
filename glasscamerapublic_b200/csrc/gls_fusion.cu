// gls_fusion.cu — pyramid burst fusion (gls_fuse_pyramid).
//
// The reference declares a pyramid fusion API but has no live
// implementation (pyramid_processor.hpp:51-55, 64-70 are commented out); its
// burst driver fuses by registerAndFuse, a running mean of pull-warped
// frames (SURF.metal:489-516, pyramidFusion.cpp:343-345). This is the
// library's own design, built to reduce to that mean:
//   * every frame is pull-warped into the reference frame (registerImage);
//   * each warped frame is decomposed into a Laplacian pyramid with the
//     denoiser's own operators: 4-tap bilinear box down-sampling
//     (downsampleImageXYZ, demosaic.metal:886-920) and the reconstruct
//     step's bilinear up-sampling (subtractNoiseImage, :922-959);
//   * per level and pixel, frames are averaged with weights
//     w = exp(-robustness |band - band_ref|^2) (the reference frame has
//     weight 1); robustness 0 gives uniform weights;
//   * the fused pyramid is collapsed with the same up-sampling.
// The operators are linear, so with uniform weights the result is the flat
// mean of the warped frames (up to float rounding): registerAndFuse's output.
#include <cmath>

#include "gls_common.cuh"
#include "gls_devbuf.h"
#include "gls_kernels.h"

namespace gls {

__device__ __forceinline__ float4 ld4f(const float* p) { return *reinterpret_cast<const float4*>(p); }

// bilinear up-sample of the coarse level at fine pixel (x, y), RGB
__device__ __forceinline__ float3 up3(const float* c, int cw, int ch, float rx, float ry, int x, int y) {
    const float u = (float(x) + 0.5f) * rx - 0.5f, v = (float(y) + 0.5f) * ry - 0.5f;
    const float fu = floorf(u), fv = floorf(v);
    const int xi = int(fu), yi = int(fv);
    const float ax = u - fu, ay = v - fv;
    auto at = [&](int X, int Y) {
        X = clampi(X, 0, cw - 1);
        Y = clampi(Y, 0, ch - 1);
        return ld4f(c + (size_t(Y) * cw + X) * 4);
    };
    const float4 a = at(xi, yi), b = at(xi + 1, yi), cc = at(xi, yi + 1), d = at(xi + 1, yi + 1);
    auto lerp2 = [&](float p, float q, float r, float s) {
        const float top = p + (q - p) * ax, bot = r + (s - r) * ax;
        return top + (bot - top) * ay;
    };
    return make_float3(lerp2(a.x, b.x, cc.x, d.x), lerp2(a.y, b.y, cc.y, d.y), lerp2(a.z, b.z, cc.z, d.z));
}

struct FuseLevelArgs {
    int w, h, cw, ch;  // level and next-coarser sizes (cw = 0: coarsest level)
    float rx, ry;
    const float *g, *gc, *rg, *rgc;  // frame and reference Gaussian levels (RGBA F32)
    float4* acc;                     // (sum w band, sum w)
    float robustness;
    int init;  // 1: this is the reference frame
};

// One band of one frame into the level's weighted sum.
__global__ void __launch_bounds__(256) k_fuse_accum(FuseLevelArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = size_t(y) * a.w + x;
    const float4 g = ld4f(a.g + i * 4);
    float3 band = make_float3(g.x, g.y, g.z);
    if (a.cw > 0) {
        const float3 u = up3(a.gc, a.cw, a.ch, a.rx, a.ry, x, y);
        band = make_float3(band.x - u.x, band.y - u.y, band.z - u.z);
    }
    if (a.init) {
        a.acc[i] = make_float4(band.x, band.y, band.z, 1.f);
        return;
    }
    float w = 1.f;
    if (a.robustness > 0.f) {
        const float4 r = ld4f(a.rg + i * 4);
        float3 rb = make_float3(r.x, r.y, r.z);
        if (a.cw > 0) {
            const float3 u = up3(a.rgc, a.cw, a.ch, a.rx, a.ry, x, y);
            rb = make_float3(rb.x - u.x, rb.y - u.y, rb.z - u.z);
        }
        const float dx = band.x - rb.x, dy = band.y - rb.y, dz = band.z - rb.z;
        w = expf(-a.robustness * (dx * dx + dy * dy + dz * dz));
    }
    const float4 c = a.acc[i];
    a.acc[i] = make_float4(c.x + w * band.x, c.y + w * band.y, c.z + w * band.z, c.w + w);
}

struct CollapseArgs {
    int w, h, cw, ch;
    float rx, ry;
    const float4* acc;
    const float* coarse;  // collapsed coarser level (RGBA F32), or null at the coarsest
    float* out;           // RGBA F32
};

__global__ void __launch_bounds__(256) k_fuse_collapse(CollapseArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = size_t(y) * a.w + x;
    const float4 c = a.acc[i];
    float3 v = make_float3(c.x / c.w, c.y / c.w, c.z / c.w);
    if (a.coarse) {
        const float3 u = up3(a.coarse, a.cw, a.ch, a.rx, a.ry, x, y);
        v = make_float3(v.x + u.x, v.y + u.y, v.z + u.z);
    }
    *reinterpret_cast<float4*>(a.out + i * 4) = make_float4(v.x, v.y, v.z, 0.f);
}

template <class O>
__global__ void k_fuse_store(const float* in, int w, int h, O* out, size_t pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float4 v = ld4f(in + (size_t(y) * w + x) * 4);
    st4<O>(out + size_t(y) * pitch + size_t(x) * 4, f4{v.x, v.y, v.z, v.w});
}

// scratch kept by the registration context between calls
struct FusionScratch {
    DevBuf ref[GLS_MAX_LEVELS], frm[GLS_MAX_LEVELS], acc[GLS_MAX_LEVELS], col[GLS_MAX_LEVELS];
    ~FusionScratch() {
        for (int l = 0; l < GLS_MAX_LEVELS; l++) {
            ref[l].release();
            frm[l].release();
            acc[l].release();
            col[l].release();
        }
    }
};

FusionScratch* fusion_scratch_new() { return new FusionScratch(); }
void fusion_scratch_delete(FusionScratch* f) { delete f; }

static inline dim3 grid2d(int w, int h) { return dim3((w + 31) / 32, (h + 7) / 8); }

gls_status fuse_pyramid_impl(FusionScratch* F, const gls_image_view* frames, int n, const float* H, int levels,
                             float robustness, gls_image_view* out, cudaStream_t s) {
    const int W = frames[0].width, Hh = frames[0].height;
    for (int l = 0; l < levels; l++) {
        const size_t bytes = size_t(W >> l) * (Hh >> l) * 16;
        GLS_TRY(F->ref[l].ensure(bytes));
        GLS_TRY(F->frm[l].ensure(bytes));
        GLS_TRY(F->acc[l].ensure(bytes));
        GLS_TRY(F->col[l].ensure(bytes));
    }
    auto lvl = [&](DevBuf* b, int l) { return Plane<float, 4>{static_cast<float*>(b[l].p), W >> l, Hh >> l,
                                                              size_t(W >> l) * 4}; };
    const dim3 blk(32, 8);
    for (int f = 0; f < n; f++) {
        DevBuf* G = f == 0 ? F->ref : F->frm;
        // pull-warp into the reference frame (identity for the reference)
        static const float I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        gls_image_view dst{G[0].p, W, Hh, 4, GLS_F32, size_t(W) * 16};
        GLS_TRY(gls_register_image(&frames[f], &dst, f == 0 ? I : H + size_t(f) * 9, s));
        for (int l = 1; l < levels; l++) launch_downsample<float, 4>(lvl(G, l - 1), lvl(G, l), s);
        for (int l = 0; l < levels; l++) {
            FuseLevelArgs a{};
            a.w = W >> l;
            a.h = Hh >> l;
            a.cw = l + 1 < levels ? (W >> (l + 1)) : 0;
            a.ch = l + 1 < levels ? (Hh >> (l + 1)) : 0;
            a.rx = a.cw ? float(a.cw) / float(a.w) : 0.f;
            a.ry = a.cw ? float(a.ch) / float(a.h) : 0.f;
            a.g = static_cast<const float*>(G[l].p);
            a.gc = a.cw ? static_cast<const float*>(G[l + 1].p) : nullptr;
            a.rg = static_cast<const float*>(F->ref[l].p);
            a.rgc = a.cw ? static_cast<const float*>(F->ref[l + 1].p) : nullptr;
            a.acc = static_cast<float4*>(F->acc[l].p);
            a.robustness = robustness;
            a.init = f == 0;
            k_fuse_accum<<<grid2d(a.w, a.h), blk, 0, s>>>(a);
        }
    }
    for (int l = levels - 1; l >= 0; l--) {
        CollapseArgs c{};
        c.w = W >> l;
        c.h = Hh >> l;
        c.cw = l + 1 < levels ? (W >> (l + 1)) : 0;
        c.ch = l + 1 < levels ? (Hh >> (l + 1)) : 0;
        c.rx = c.cw ? float(c.cw) / float(c.w) : 0.f;
        c.ry = c.cw ? float(c.ch) / float(c.h) : 0.f;
        c.acc = static_cast<const float4*>(F->acc[l].p);
        c.coarse = c.cw ? static_cast<const float*>(F->col[l + 1].p) : nullptr;
        c.out = static_cast<float*>(F->col[l].p);
        k_fuse_collapse<<<grid2d(c.w, c.h), blk, 0, s>>>(c);
    }
    const size_t es = out->dtype == GLS_F32 ? 4 : 2;
    const size_t pitch = (out->stride_bytes ? out->stride_bytes : size_t(W) * 4 * es) / es;
    if (out->dtype == GLS_F32)
        k_fuse_store<float><<<grid2d(W, Hh), blk, 0, s>>>(static_cast<const float*>(F->col[0].p), W, Hh,
                                                           static_cast<float*>(out->data), pitch);
    else
        k_fuse_store<__half><<<grid2d(W, Hh), blk, 0, s>>>(static_cast<const float*>(F->col[0].p), W, Hh,
                                                            static_cast<__half*>(out->data), pitch);
    GLS_CUDA(cudaGetLastError());
    return GLS_OK;
}

}  // namespace gls
