// gls_post.cu — display post-processing of RawConverter::demosaic with
// postProcess (raw_converter.cpp:80-116, 224-244):
//   * k_hist / k_hist_stats   histogramImage + histogramStatistics
//                             (demosaic.metal:1373-1455) on the luma of the
//                             denoised level 3: per-block shared-memory
//                             counts, then one thread for the statistics in
//                             the reference's float order (exact thresholds)
//   * k_noise_tables          the grain tables from the raw frame's first
//                             pixel (gls_noise.h), on the device
//   * k_guided_box            GuidedFilterABImage + BoxFilterGFImage
//                             (:1295-1356) fused per band: the 5x5 (a, b)
//                             of a tile plus halo in shared memory, then the
//                             9-tap box, so the full-resolution (a, b) plane
//                             never reaches HBM
//   * k_post_srgb             transformImage to camera RGB,
//                             localToneMappingMaskImage (:1481-1544) and
//                             convertTosRGB (:1621-1705) fused per pixel
// Sampling conventions: the guided filter and box taps at their texel
// positions, clamp-to-edge; each band's (a, b) read bilinearly at
// (x + 0.5) * (band size / size) - 0.5.
#include <cfloat>
#include <cmath>
#include <cstring>

#include "../../include/glscam.h"
#include "gls_common.cuh"
#include "gls_fmath.h"
#include "gls_kernels.h"
#include "gls_noise.h"

namespace gls {

namespace {

// ---------------------------------------------------------------- histogram
template <class S>
__global__ void __launch_bounds__(256) k_hist(Plane<S, 4> img, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    h[tid] = 0;
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < img.w && y < img.h) {
        const float v = ld4<S>(img.px(x, y)).x;
        const int idx = clampi(int(__fmul_rn(255.0f, __fsqrt_rn(__fdiv_rn(v, 2.0f)))), 0, 255);
        atomicAdd(&h[idx], 1u);
    }
    __syncthreads();
    if (h[tid]) atomicAdd(&hist[tid], h[tid]);
}

__device__ __forceinline__ float sstep_rn(float e0, float e1, float x) {  // smoothstep, one rounding per op
    using namespace glsm;
    const float t = fminf(fmaxf(fdiv(fsub(x, e0), fsub(e1, e0)), 0.0f), 1.0f);
    return fmul(fmul(t, t), fsub(3.0f, fmul(2.0f, t)));
}

// histogramStatistics, one thread; fixed != 0: the levels the reference
// sets without noise reduction (raw_converter.cpp:224-229)
__global__ void k_hist_stats(const uint32_t* __restrict__ hist, uint32_t image_size, int fixed, PostStats* st) {
    using namespace glsm;
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    PostStats s{};
    if (fixed) {
        s.black = 0.1f;
        s.white = 1.0f;
        s.mean = 0.22f;
        s.median = 0.22f;
        *st = s;
        return;
    }
    uint32_t bands[8] = {};
    float mean = 0.0f;
    bool found_median = false, found_black = false, found_white = false;
    int median_index = 0, black_index = 0, white_index = 0;
    uint32_t sum = 0;
    for (int band = 0; band < 8; band++)
        for (int i = 0; i < 32; i++) {
            const int index = band * 32 + i;
            const uint32_t entry = hist[index];
            bands[band] += entry;
            mean = fadd(mean, fdiv(float(entry * uint32_t(index + 1)), 256.0f));
            sum += entry;
            if (!found_median && sum >= (image_size + 1) / 2) {
                median_index = index;
                found_median = true;
            }
            if (!found_black && float(sum) >= fmul(0.001f, float(image_size))) {
                black_index = index;
                found_black = true;
            }
            if (!found_white && float(sum) >= fmul(0.999f, float(image_size))) {
                white_index = index;
                found_white = true;
            }
        }
    mean = fdiv(mean, float(image_size));
    {
        const float v = fdiv(float(black_index - 1), 255.0f);
        s.black = fmul(fmul(2.0f, v), v);
    }
    {
        const float v = fdiv(float(white_index), 255.0f);
        s.white = fmul(fmul(2.0f, v), v);
    }
    s.median = fsub(fdiv(float(median_index), 255.0f), s.black);
    s.mean = fsub(mean, s.black);
    s.highlights = fadd(1.0f, fmul(2.0f, sstep_rn(0.01f, 0.1f, fdiv(float(bands[5] + bands[6] + bands[7]),
                                                                     float(image_size)))));
    s.shadows = fsub(0.8f, fmul(0.5f, sstep_rn(0.25f, 0.5f, fdiv(float(bands[0] + bands[1]), float(image_size)))));
    *st = s;
}

__global__ void k_noise_tables(const uint16_t* __restrict__ raw, int* __restrict__ perm, float* __restrict__ grad) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    noise_tables(uint32_t(raw[0]), perm, grad);
}

// ---------------------------------------------------------------- LTM bands
constexpr int GB_TX = 32, GB_TY = 8;
constexpr int GB_AW = GB_TX + 4, GB_AH = GB_TY + 4;  // (a, b) tile: halo 2 for the box
constexpr int GB_GW = GB_AW + 4, GB_GH = GB_AH + 4;  // guide tile: halo 2 more for the 5x5 window

template <class S>
__global__ void __launch_bounds__(GB_TX * GB_TY) k_guided_box(Plane<S, 4> guide, float eps, float2* __restrict__ out) {
    __shared__ float gy[GB_GH][GB_GW];
    __shared__ float2 ab[GB_AH][GB_AW];
    const int x0 = blockIdx.x * GB_TX, y0 = blockIdx.y * GB_TY;
    const int tid = threadIdx.y * GB_TX + threadIdx.x, nt = GB_TX * GB_TY;
    const int W = guide.w, H = guide.h;
    // guide luma around the (a, b) positions; (a, b) is computed at the
    // clamped position of each halo entry, as a clamp-to-edge read of the
    // reference's (a, b) texture returns it
    for (int k = tid; k < GB_GW * GB_GH; k += nt) {
        const int ty = k / GB_GW, tx = k % GB_GW;
        gy[ty][tx] = ld4<S>(guide.pxc(x0 - 4 + tx, y0 - 4 + ty)).x;  // unused entries near clamped edges stay harmless
    }
    __syncthreads();
    for (int k = tid; k < GB_AW * GB_AH; k += nt) {
        const int ty = k / GB_AW, tx = k % GB_AW;
        const int px = clampi(x0 - 2 + tx, 0, W - 1), py = clampi(y0 - 2 + ty, 0, H - 1);
        float sum = 0.f, sumSq = 0.f;
        for (int dy = -2; dy <= 2; dy++)
            for (int dx = -2; dx <= 2; dx++) {
                // the guide at clamp(p + d): inside the staged tile whenever p is,
                // else read directly
                const int qx = clampi(px + dx, 0, W - 1), qy = clampi(py + dy, 0, H - 1);
                const int lx = qx - (x0 - 4), ly = qy - (y0 - 4);
                const float s = (lx >= 0 && lx < GB_GW && ly >= 0 && ly < GB_GH) ? gy[ly][lx]
                                                                                 : ld4<S>(guide.px(qx, qy)).x;
                sum += s;
                sumSq += s * s;
            }
        const float mean = sum / 25.f;
        const float var = (sumSq - sum * sum / 25.f) / 25.f;
        const float a = var / (var + eps);
        ab[ty][tx] = make_float2(a, mean * (1.f - a));
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= W || y >= H) return;
    // nine bilinear taps: offsets -1.5 and 0.5 average two neighbours, 2.0
    // is one texel (BoxFilterGFImage's table)
    const float w[9] = {0.16f, 0.16f, 0.08f, 0.16f, 0.16f, 0.08f, 0.08f, 0.08f, 0.04f};
    const int ox[9] = {-2, 0, 2, -2, 0, 2, -2, 0, 2}, oy[9] = {-2, -2, -2, 0, 0, 0, 2, 2, 2};
    const bool hx[9] = {true, true, false, true, true, false, true, true, false};
    const bool hy[9] = {true, true, true, true, true, true, false, false, false};
    const int cx = threadIdx.x + 2, cy = threadIdx.y + 2;
    float2 m = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 9; i++) {
        auto tap = [&](int dx, int dy) { return ab[cy + dy][cx + dx]; };
        float2 top, bot;
        const float2 a00 = tap(ox[i], oy[i]);
        const float2 a01 = hx[i] ? tap(ox[i] + 1, oy[i]) : a00;
        top = make_float2(a00.x + (a01.x - a00.x) * (hx[i] ? 0.5f : 0.f), a00.y + (a01.y - a00.y) * (hx[i] ? 0.5f : 0.f));
        if (hy[i]) {
            const float2 a10 = tap(ox[i], oy[i] + 1);
            const float2 a11 = hx[i] ? tap(ox[i] + 1, oy[i] + 1) : a10;
            bot = make_float2(a10.x + (a11.x - a10.x) * (hx[i] ? 0.5f : 0.f),
                              a10.y + (a11.y - a10.y) * (hx[i] ? 0.5f : 0.f));
            top = make_float2(top.x + (bot.x - top.x) * 0.5f, top.y + (bot.y - top.y) * 0.5f);
        }
        m.x += w[i] * top.x;
        m.y += w[i] * top.y;
    }
    out[size_t(y) * W + x] = m;
}

// ---------------------------------------------------------------- per pixel
struct Band {
    const float2* ab;
    int w, h;
    float rx, ry;  // band size / image size
};

struct SrgbArgs {
    float m[9];        // YCbCr -> camera RGB (with input_ycc)
    float rgb_cam[9];  // convertTosRGB's transform
    float contrast, saturation, slope, bias_mul, blacks;
    int ltm, input_ycc;
    float detail[3];
    float nlf[2], luma_var[2];
    Band band[3];
};

__device__ __forceinline__ float sstep(float e0, float e1, float x) { return smoothstepf(e0, e1, x); }

__device__ __forceinline__ float2 band_ab(const Band& b, int x, int y) {
    const float u = (float(x) + 0.5f) * b.rx - 0.5f, v = (float(y) + 0.5f) * b.ry - 0.5f;
    const float fu = floorf(u), fv = floorf(v);
    const int xi = int(fu), yi = int(fv);
    const float ax = u - fu, ay = v - fv;
    auto at = [&](int X, int Y) { return b.ab[size_t(clampi(Y, 0, b.h - 1)) * b.w + clampi(X, 0, b.w - 1)]; };
    const float2 p00 = at(xi, yi), p01 = at(xi + 1, yi), p10 = at(xi, yi + 1), p11 = at(xi + 1, yi + 1);
    const float tx = p00.x + (p01.x - p00.x) * ax, bx = p10.x + (p11.x - p10.x) * ax;
    const float ty = p00.y + (p01.y - p00.y) * ax, by = p10.y + (p11.y - p10.y) * ax;
    return make_float2(tx + (bx - tx) * ay, ty + (by - ty) * ay);
}

__device__ __forceinline__ float ltm_multiplier(float Y, float ill, float shadows, float highlights, float detail) {
    const float mid = 0.22f, rest = 1.f - 0.22f;
    const float refl = Y / ill;
    const float adj = ill <= mid ? mid * powf(ill / mid, shadows) : rest * powf((ill - mid) / rest, highlights) + mid;
    return adj * powf(refl, detail) / Y;
}

__device__ __forceinline__ float noise2(const int* __restrict__ P, const float2* __restrict__ G, float px, float py) {
    const float tx = px + 4096.0f, ty = py + 4096.0f;
    const int b0x = int(tx) & 255, b0y = int(ty) & 255;
    const int b1x = (b0x + 1) & 255, b1y = (b0y + 1) & 255;
    const float r0x = tx - floorf(tx), r0y = ty - floorf(ty);
    const float r1x = r0x - 1.f, r1y = r0y - 1.f;
    const int i = P[b0x], j = P[b1x];
    const int b00 = P[i + b0y], b10 = P[j + b0y], b01 = P[i + b1y], b11 = P[j + b1y];
    const float sx = r0x * r0x * (3.f - 2.f * r0x), sy = r0y * r0y * (3.f - 2.f * r0y);
    auto dot2 = [&](int g, float ax, float ay) { return G[g].x * ax + G[g].y * ay; };
    float u = dot2(b00, r0x, r0y), v = dot2(b10, r1x, r0y);
    const float a = u + (v - u) * sx;
    u = dot2(b01, r0x, r1y);
    v = dot2(b11, r1x, r1y);
    const float b = u + (v - u) * sx;
    return a + (b - a) * sy;
}

__device__ __forceinline__ float octave_noise(const int* P, const float2* G, float px, float py) {
    float freq = 1.f, amp = 1.f, norm = 1.f;
    float sum = noise2(P, G, px, py);
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        freq *= 0.5f;
        amp *= 0.5f;
        norm += amp;
        sum += noise2(P, G, px * freq, py * freq) * amp;
    }
    return sum / norm;
}

__device__ __forceinline__ float sigmoid(float x, float s) { return 0.5f * (tanhf(s * x - 0.3f * s) + 1.f); }
__device__ __forceinline__ float tone_curve(float x, float s) {
    return (sigmoid(powf(0.95f * x, 0.5f), s) - sigmoid(0.f, s)) / (sigmoid(1.f, s) - sigmoid(0.f, s));
}

template <class S, class O>
__global__ void __launch_bounds__(256) k_post_srgb(Plane<S, 4> in, Plane<S, 2> grad, const PostStats* __restrict__ st_,
                                                   const int* __restrict__ perm, const float2* __restrict__ gtab,
                                                   SrgbArgs a, Plane<O, 4> out) {
    __shared__ int P[kNoiseSize];
    __shared__ float2 G[kNoiseSize];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int k = tid; k < kNoiseSize; k += blockDim.x * blockDim.y) {
        P[k] = perm[k];
        G[k] = gtab[k];
    }
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= in.w || y >= in.h) return;
    const PostStats st = *st_;
    const f4 p = ld4<S>(in.px(x, y));
    float rin[3];
    if (a.input_ycc) {  // transformImage YCbCr -> camera RGB (raw_converter.cpp:219)
        rin[0] = a.m[0] * p.x + a.m[1] * p.y + a.m[2] * p.z;
        rin[1] = a.m[3] * p.x + a.m[4] * p.y + a.m[5] * p.z;
        rin[2] = a.m[6] * p.x + a.m[7] * p.y + a.m[8] * p.z;
    } else {
        rin[0] = p.x;
        rin[1] = p.y;
        rin[2] = p.z;
    }
    // ---- localToneMappingMaskImage
    float mask = 1.f;
    if (a.ltm) {
        const float Y = p.x;
        for (int k = 0; k < 3; k++) {
            const float2 abk = band_ab(a.band[k], x, y);
            const float ill = abk.x * Y + abk.y;
            float d = a.detail[k];
            if (d > 1.f) {
                float dd = (1.f - sstep(0.75f, 0.95f, ill)) * sstep(0.05f, 0.1f, ill);
                if (k == 2) {
                    const f2 g = ld2<S>(grad.px(x, y));
                    const float gl = sqrtf(g.x * g.x + g.y * g.y);
                    const float sigma = sqrtf(a.nlf[0] + a.nlf[1] * ill);
                    dd = sstep(2.f * sigma, 8.f * sigma, gl) * (1.f - sstep(32.f * sigma, 128.f * sigma, gl)) * dd;
                }
                d = 1.f + (d - 1.f) * dd;
            }
            mask *= ltm_multiplier(Y, ill, st.shadows, k == 0 ? st.highlights : 1.f, d);
        }
    }
    // ---- convertTosRGB
    const float black = st.black, white = 1.f;
    float brightening = 1.f;
    if (st.mean > 0.22f) brightening *= 0.22f / st.mean;
    float pv[3];
    for (int c = 0; c < 3; c++) pv[c] = brightening * fmaxf(rin[c] - black, 0.f) / (white - black) * a.bias_mul;
    if (a.saturation != 1.f) {
        const float luma = 0.2126f * pv[0] + 0.7152f * pv[1] + 0.0722f * pv[2];
        for (int c = 0; c < 3; c++) pv[c] = mixf(luma, pv[c], mixf(a.saturation, 1.f, sstep(0.75f, 2.f, pv[c])));
    }
    if (a.contrast != 1.f)
        for (int c = 0; c < 3; c++) pv[c] = mixf(0.2f, pv[c], mixf(a.contrast, 1.f, sstep(0.9f, 2.f, pv[c])));
    float rgb[3];
    for (int c = 0; c < 3; c++)
        rgb[c] = fmaxf(a.rgb_cam[3 * c] * pv[0] + a.rgb_cam[3 * c + 1] * pv[1] + a.rgb_cam[3 * c + 2] * pv[2], 0.f);
    float sigma = 0.f;
    const bool lv = a.luma_var[0] != 0.f || a.luma_var[1] != 0.f;
    if (a.ltm) {
        if (mask > 1.f) {
            const float luma = 0.2126f * rgb[0] + 0.7152f * rgb[1] + 0.0722f * rgb[2];
            const float t = fminf(powf(luma, 0.5f), 1.f), s = sstep(0.5f, 0.8f, luma);
            for (int c = 0; c < 3; c++) {
                const float lifted = 1.f - (1.f - rgb[c]) * (1.f - mask * luma) / (1.f - luma);
                rgb[c] = mixf(rgb[c] * mask, mixf(lifted, rgb[c] * mask, s), t);
            }
        } else if (mask < 1.f) {
            for (int c = 0; c < 3; c++) rgb[c] *= mask;
        }
        if (lv) sigma = sqrtf(a.luma_var[0] + a.luma_var[1] * mask * rin[1]);
    } else if (lv) {
        sigma = sqrtf(a.luma_var[0] + a.luma_var[1] * rin[1]);
    }
    if (sigma > 0.f) {
        const float n = octave_noise(P, G, 0.5f * float(x), 0.5f * float(y));
        for (int c = 0; c < 3; c++) rgb[c] += sigma * n;
    }
    f4 o;
    float* ov = &o.x;
    for (int c = 0; c < 3; c++) {
        float v = tone_curve(fmaxf(rgb[c], 0.f), a.slope);
        if (a.blacks > 0.f) v = (v - a.blacks) / (1.f - a.blacks);
        ov[c] = clampf(v, 0.f, 1.f);
    }
    o.w = 1.f;
    st4<O>(out.px(x, y), o);
}

}  // namespace

size_t post_ab_bytes(int w, int h) {
    return (size_t(w >> 4) * (h >> 4) + size_t(w >> 2) * (h >> 2) + size_t(w) * h) * sizeof(float2);
}

template <class S, class O>
void launch_post(const PostArgs<S>& pa, Plane<O, 4> out, cudaStream_t s) {
    const dim3 b(32, 8);
    auto grid = [&](int w, int h) { return dim3((w + 31) / 32, (h + 7) / 8); };
    cudaMemsetAsync(pa.hist, 0, 256 * sizeof(uint32_t), s);
    if (pa.denoise) k_hist<S><<<grid(pa.den[3].w, pa.den[3].h), b, 0, s>>>(pa.den[3], pa.hist);
    k_hist_stats<<<1, 32, 0, s>>>(pa.hist, uint32_t(pa.den[3].w) * uint32_t(pa.den[3].h), pa.denoise ? 0 : 1,
                                  pa.stats);
    k_noise_tables<<<1, 32, 0, s>>>(pa.raw, pa.perm, pa.grad_tab);
    SrgbArgs a{};
    const gls_demosaic_params& p = *pa.params;
    std::memcpy(a.m, pa.y2c, sizeof(a.m));
    std::memcpy(a.rgb_cam, p.rgb_cam, sizeof(a.rgb_cam));
    a.contrast = p.rgb_conversion.contrast;
    a.saturation = p.rgb_conversion.saturation;
    a.slope = p.rgb_conversion.tone_curve_slope;
    // exposureBias += log2(exposure_multiplier) (raw_converter.cpp:235)
    const float bias = p.rgb_conversion.exposure_bias + std::log2(p.exposure_multiplier);
    a.bias_mul = bias != 0.f ? std::pow(2.0f, bias) : 1.f;
    a.blacks = p.rgb_conversion.blacks;
    a.ltm = (pa.denoise && p.rgb_conversion.local_tone_mapping) ? 1 : 0;
    a.input_ycc = pa.denoise ? 1 : 0;
    for (int k = 0; k < 3; k++) a.detail[k] = p.ltm.detail[k];
    a.nlf[0] = p.pyramid_nlf[0].a[0];
    a.nlf[1] = p.pyramid_nlf[0].b[0];
    a.luma_var[0] = 2.0f * ((p.raw_nlf.a[1] + p.raw_nlf.a[3]) / 2);
    a.luma_var[1] = 2.0f * ((p.raw_nlf.b[1] + p.raw_nlf.b[3]) / 2);
    const Plane<S, 4>& in = pa.denoise ? pa.den[0] : pa.rgb;
    if (a.ltm) {  // guides: denoised levels 4, 2, 0 (raw_converter.cpp:105-110)
        const int lv[3] = {4, 2, 0};
        float2* ab = pa.ab;
        for (int k = 0; k < 3; k++) {
            const Plane<S, 4>& g = pa.den[lv[k]];
            k_guided_box<S><<<dim3((g.w + GB_TX - 1) / GB_TX, (g.h + GB_TY - 1) / GB_TY), dim3(GB_TX, GB_TY), 0, s>>>(
                g, p.ltm.eps, ab);
            a.band[k] = {ab, g.w, g.h, float(g.w) / float(in.w), float(g.h) / float(in.h)};
            ab += size_t(g.w) * g.h;
        }
    }
    k_post_srgb<S, O><<<grid(in.w, in.h), b, 0, s>>>(in, pa.grad2, pa.stats, pa.perm,
                                                       reinterpret_cast<const float2*>(pa.grad_tab), a, out);
}

template void launch_post<float, float>(const PostArgs<float>&, Plane<float, 4>, cudaStream_t);
template void launch_post<float, __half>(const PostArgs<float>&, Plane<__half, 4>, cudaStream_t);
template void launch_post<__half, float>(const PostArgs<__half>&, Plane<float, 4>, cudaStream_t);
template void launch_post<__half, __half>(const PostArgs<__half>&, Plane<__half, 4>, cudaStream_t);

}  // namespace gls
