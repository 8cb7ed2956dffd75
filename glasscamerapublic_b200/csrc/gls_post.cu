// gls_post.cu — display post-processing of RawConverter::demosaic with
// postProcess (raw_converter.cpp:80-116, 224-244):
//   * k_hist                  histogramImage (demosaic.metal:1373-1383) on
//                             the luma of the denoised level 3: per-block
//                             shared-memory counts added to the histogram
//   * k_post_tables           one block: warp 0 runs histogramStatistics
//                             (:1385-1455) in the reference's float order
//                             (exact thresholds) and zeroes the histogram for
//                             the next frame; warp 1 draws the grain tables
//                             from the raw frame's first pixel (gls_noise.h)
//   * k_guided_box            GuidedFilterABImage + BoxFilterGFImage
//                             (:1295-1356) fused, the three bands in one
//                             launch: the 5x5 (a, b) of a tile plus halo in
//                             shared memory, then the 9-tap box, so the
//                             unfiltered (a, b) planes never reach HBM
//   * k_post_srgb             transformImage to camera RGB,
//                             localToneMappingMaskImage (:1481-1544) and
//                             convertTosRGB (:1621-1705) fused per pixel
// Sampling conventions: the guided filter and box taps at their texel
// positions, clamp-to-edge; each band's (a, b) read bilinearly at
// (x + 0.5) * (band size / size) - 0.5.
// Arithmetic (FP32), in the fast-math style the reference's Metal kernels
// compile to: pow(x, y) as exp2(y log2 x) on the hardware's base-2
// logarithm and exponential, with log2 of the luma shared by the three
// tone-mapping bands; square roots and the per-pixel divisions by the
// hardware's approximations (relative error about 2^-22); the sigmoid as a
// logistic of exp2; smoothstep by the reciprocal of its edge span; the
// tone curve's end points once per launch on the host. The guided filter's
// 5x5 sums are column sums then row sums. A thread converts four rows of a 32 x 32
// tile, so a block stages the grain tables once per 1024 pixels.
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

// histogramStatistics and the grain tables in one block of 256 threads;
// fixed != 0: the levels the reference sets without noise reduction
// (raw_converter.cpp:224-229). The histogram is left zeroed for the next
// frame (the buffer is zeroed when allocated).
//   * statistics: each thread forms its bin's mean term (exact: a count
//     times (index + 1), over 256); thread 0 then runs the reference's scan
//     in its order (demosaic.metal:1397-1423);
//   * grain tables: thread 32 steps the C library's random() (gls_noise.h)
//     with its 34-entry ring in registers (groups of 34 steps keep every ring
//     index static), writing the 767 outputs initGradients draws to shared
//     memory; all threads then form and normalise the gradients, and
//     thread 0 runs the Fisher-Yates shuffle (SimplexNoise.hpp:109-130).
constexpr int kRandDiscard = 310, kRandUsed = 2 * 256 + 255;

__device__ void random_outputs(uint32_t seed, int* __restrict__ outs) {
    uint32_t r[34];
    int32_t word = seed == 0 ? 1 : int32_t(seed);
    r[0] = uint32_t(word);
#pragma unroll
    for (int k = 1; k < 31; k++) {
        const int32_t hi = word / 127773, lo = word % 127773;
        word = 16807 * lo - 2836 * hi;
        if (word < 0) word += 2147483647;
        r[k] = uint32_t(word);
    }
#pragma unroll
    for (int k = 31; k < 34; k++) r[k] = r[k - 31];
    // step n writes ring slot n % 34 from slots (n + 3) % 34 and (n + 31) % 34
    constexpr int total = kRandDiscard + kRandUsed;
#pragma unroll 1
    for (int n0 = 0; n0 < total; n0 += 34) {
#pragma unroll
        for (int j = 0; j < 34; j++) {
            const int n = n0 + j;
            if (n < total) {
                const uint32_t v = r[(j + 3) % 34] + r[(j + 31) % 34];
                r[j] = v;
                if (n >= kRandDiscard) outs[n - kRandDiscard] = int32_t(v >> 1);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_post_tables(uint32_t* __restrict__ hist, uint32_t image_size, int fixed,
                                                     PostStats* __restrict__ st, const uint16_t* __restrict__ raw,
                                                     int* __restrict__ perm, float* __restrict__ grad) {
    using namespace glsm;
    __shared__ uint32_t h[256];
    __shared__ float term[256];
    __shared__ int outs[kRandUsed];
    __shared__ int P[256];
    const int t = threadIdx.x;
    h[t] = hist[t];
    hist[t] = 0;
    term[t] = fdiv(float(h[t] * uint32_t(t + 1)), 256.0f);
    P[t] = t;
    __syncthreads();
    if (t == 0) {
        PostStats s{};
        if (fixed) {
            s.black = 0.1f;
            s.white = 1.0f;
            s.mean = 0.22f;
            s.median = 0.22f;
        } else {
            uint32_t bands[8] = {};
            float mean = 0.0f;
            bool found_median = false, found_black = false, found_white = false;
            int median_index = 0, black_index = 0, white_index = 0;
            uint32_t sum = 0;
            const float black_at = fmul(0.001f, float(image_size)), white_at = fmul(0.999f, float(image_size));
            for (int index = 0; index < 256; index++) {
                const uint32_t entry = h[index];
                bands[index >> 5] += entry;
                mean = fadd(mean, term[index]);
                sum += entry;
                if (!found_median && sum >= (image_size + 1) / 2) {
                    median_index = index;
                    found_median = true;
                }
                if (!found_black && float(sum) >= black_at) {
                    black_index = index;
                    found_black = true;
                }
                if (!found_white && float(sum) >= white_at) {
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
            s.shadows =
                fsub(0.8f, fmul(0.5f, sstep_rn(0.25f, 0.5f, fdiv(float(bands[0] + bands[1]), float(image_size)))));
        }
        *st = s;
    } else if (t == 32) {
        random_outputs(uint32_t(raw[0]), outs);
    }
    __syncthreads();
    {  // gradient t: two draws, each (r % 512 - 256) / 256, normalised
        const float gx = float((outs[2 * t] % 512) - 256) / 256, gy = float((outs[2 * t + 1] % 512) - 256) / 256;
        const float n = sqrtf(gx * gx + gy * gy);
        const float2 g = make_float2(gx / n, gy / n);
        reinterpret_cast<float2*>(grad)[t] = g;
        reinterpret_cast<float2*>(grad)[256 + t] = g;
        if (t < 2) reinterpret_cast<float2*>(grad)[512 + t] = g;
    }
    if (t == 0) {
        for (int i = 255; i > 0; i--) {
            const int k = P[i];
            const int j = outs[512 + (255 - i)] % 256;
            P[i] = P[j];
            P[j] = k;
        }
    }
    __syncthreads();
    perm[t] = P[t];
    perm[256 + t] = P[t];
    if (t < 2) perm[512 + t] = P[t];
}

// ---------------------------------------------------------------- LTM bands
// A block of 32 x 8 threads filters a 32 x 16 tile (two rows per thread).
constexpr int GB_TX = 32, GB_TY = 8, GB_OY = 16;
constexpr int GB_AW = GB_TX + 4, GB_AH = GB_OY + 4;  // (a, b) tile: halo 2 for the box
constexpr int GB_GW = GB_AW + 4, GB_GH = GB_AH + 4;  // guide tile: halo 2 more for the 5x5 window

// the three bands of one launch: blocks [first[k], first[k + 1]) tile band k
template <class S>
struct GuideBands {
    Plane<S, 4> guide[3];
    float2* out[3];
    int tiles_x[3];
    int first[4];
};

template <class S>
__global__ void __launch_bounds__(GB_TX * GB_TY) k_guided_box(GuideBands<S> gb, float eps) {
    __shared__ float gy[GB_GH][GB_GW];
    __shared__ float2 cs[GB_AH][GB_GW];  // 5-row column sums of (v, v^2)
    __shared__ float2 ab[GB_AH][GB_AW];
    const int blk = blockIdx.x;
    // the band by selects, not by a run-time index into the parameter arrays
    // (which would copy them to local memory)
    const bool b0 = blk < gb.first[1], b1 = !b0 && blk < gb.first[2];
    const Plane<S, 4> guide = b0 ? gb.guide[0] : (b1 ? gb.guide[1] : gb.guide[2]);
    float2* __restrict__ out = b0 ? gb.out[0] : (b1 ? gb.out[1] : gb.out[2]);
    const int tiles_x = b0 ? gb.tiles_x[0] : (b1 ? gb.tiles_x[1] : gb.tiles_x[2]);
    const int t = blk - (b0 ? gb.first[0] : (b1 ? gb.first[1] : gb.first[2]));
    const int x0 = (t % tiles_x) * GB_TX, y0 = (t / tiles_x) * GB_OY;
    const int tid = threadIdx.y * GB_TX + threadIdx.x, nt = GB_TX * GB_TY;
    const int W = guide.w, H = guide.h;
    // guide luma at the clamped coordinates of the tile plus a halo of 4
    for (int k = tid; k < GB_GW * GB_GH; k += nt) {
        const int ty = k / GB_GW, tx = k % GB_GW;
        gy[ty][tx] = ld4<S>(guide.pxc(x0 - 4 + tx, y0 - 4 + ty)).x;
    }
    __syncthreads();
    // the 5x5 window sums of (a, b) over the tile plus a halo of 2, as
    // column sums then row sums: the window of position p reads gy at
    // p + d, which holds the guide at clamp(p + d)
    for (int k = tid; k < GB_GW * GB_AH; k += nt) {
        const int ty = k / GB_GW, tx = k % GB_GW;
        float sum = 0.f, sumSq = 0.f;
#pragma unroll
        for (int dy = 0; dy < 5; dy++) {
            const float v = gy[ty + dy][tx];
            sum += v;
            sumSq += v * v;
        }
        cs[ty][tx] = make_float2(sum, sumSq);
    }
    __syncthreads();
    for (int k = tid; k < GB_AW * GB_AH; k += nt) {
        const int ty = k / GB_AW, tx = k % GB_AW;
        float sum = 0.f, sumSq = 0.f;
#pragma unroll
        for (int dx = 0; dx < 5; dx++) {
            const float2 c = cs[ty][tx + dx];
            sum += c.x;
            sumSq += c.y;
        }
        const float mean = sum / 25.f;
        const float var = (sumSq - sum * sum / 25.f) / 25.f;
        const float a = var / (var + eps);
        ab[ty][tx] = make_float2(a, mean * (1.f - a));
    }
    __syncthreads();
    // a halo entry outside the image takes the (a, b) of its clamped
    // position (always inside the image and the tile), as a clamp-to-edge
    // read of the reference's (a, b) texture returns it
    if (x0 < 2 || y0 < 2 || x0 + GB_TX + 2 > W || y0 + GB_OY + 2 > H) {
        for (int k = tid; k < GB_AW * GB_AH; k += nt) {
            const int ty = k / GB_AW, tx = k % GB_AW;
            const int px = x0 - 2 + tx, py = y0 - 2 + ty;
            const int cx = clampi(px, 0, W - 1), cy = clampi(py, 0, H - 1);
            if (cx != px || cy != py) ab[ty][tx] = ab[cy - (y0 - 2)][cx - (x0 - 2)];
        }
        __syncthreads();
    }
    const int x = x0 + threadIdx.x;
    if (x >= W) return;
    // nine bilinear taps: offsets -1.5 and 0.5 average two neighbours, 2.0
    // is one texel (BoxFilterGFImage's table)
    const float w[9] = {0.16f, 0.16f, 0.08f, 0.16f, 0.16f, 0.08f, 0.08f, 0.08f, 0.04f};
    const int ox[9] = {-2, 0, 2, -2, 0, 2, -2, 0, 2}, oy[9] = {-2, -2, -2, 0, 0, 0, 2, 2, 2};
    const bool hx[9] = {true, true, false, true, true, false, true, true, false};
    const bool hy[9] = {true, true, true, true, true, true, false, false, false};
    const int cx = threadIdx.x + 2;
#pragma unroll
    for (int r = 0; r < GB_OY / GB_TY; r++) {
        const int y = y0 + threadIdx.y + r * GB_TY;
        if (y >= H) return;
        const int cy = threadIdx.y + r * GB_TY + 2;
        float2 m = make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < 9; i++) {
            auto tap = [&](int dx, int dy) { return ab[cy + dy][cx + dx]; };
            float2 top, bot;
            const float2 a00 = tap(ox[i], oy[i]);
            const float2 a01 = hx[i] ? tap(ox[i] + 1, oy[i]) : a00;
            top = make_float2(a00.x + (a01.x - a00.x) * (hx[i] ? 0.5f : 0.f),
                              a00.y + (a01.y - a00.y) * (hx[i] ? 0.5f : 0.f));
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
}

// ---------------------------------------------------------------- per pixel
struct Band {
    const float2* ab;
    int w, h;
    float rx, ry;  // band size / image size
    int full;      // the band at the image's own size: (a, b) read at the pixel
};

struct SrgbArgs {
    float m[9];        // YCbCr -> camera RGB (with input_ycc)
    float rgb_cam[9];  // convertTosRGB's transform
    float contrast, saturation, slope, bias_mul, blacks;
    float sig0, sig_rrange;  // sigmoid(0, slope) and 1 / (sigmoid(1, slope) - sigmoid(0, slope))
    int ltm, input_ycc;
    float detail[3];
    float nlf[2], luma_var[2];
    Band band[3];
};

constexpr int PS_ROWS = 4;  // rows per thread: a block of 32 x 8 threads covers 32 x 32 pixels

// smoothstep(e0, e1, x) given r = 1 / (e1 - e0)
__device__ __forceinline__ float sstep_r(float e0, float r, float x) {
    const float t = clampf((x - e0) * r, 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}
constexpr float kR_075_095 = 1.f / (0.95f - 0.75f);
constexpr float kR_005_010 = 1.f / (0.1f - 0.05f);
constexpr float kR_075_200 = 1.f / (2.f - 0.75f);
constexpr float kR_090_200 = 1.f / (2.f - 0.9f);
constexpr float kR_050_080 = 1.f / (0.8f - 0.5f);

// the hardware's square root and base-2 exponential approximations
// (relative errors about 2^-23 and 2^-22)
__device__ __forceinline__ float sqrt_a(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float ex2_a(float x) {
    float r;
    asm("ex2.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// x^y as exp2(y log2 |x|) on the hardware's base-2 logarithm and
// exponential, with pow's results for y = 0 and 1 and for negative bases
// (defined for integer y, negative for odd y)
__device__ __forceinline__ float pow_e(float x, float y) {
    if (y == 1.f) return x;
    if (y == 0.f) return 1.f;
    float r = ex2_a(y * __log2f(fabsf(x)));
    if (x < 0.f) {
        if (truncf(y) != y) return __int_as_float(0x7fc00000);
        if (fmodf(y, 2.f) != 0.f) r = -r;
    }
    return r;
}

__device__ __forceinline__ float2 band_ab(const Band& b, int x, int y) {
    if (b.full) return b.ab[size_t(y) * b.w + x];  // u = x exactly: no interpolation
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

// computeLtmMultiplier (demosaic.metal:1457-1472) times Y: the caller
// multiplies by 1 / Y, formed once for the three bands. With Y and the
// illuminance positive (lY = log2 Y) the powers are exp2 of log2
// differences and no division remains; otherwise pow's general cases.
__device__ __forceinline__ float ltm_multiplier_y(float Y, float lY, float ill, float shadows, float highlights,
                                                  float detail) {
    constexpr float mid = 0.22f, rest = 1.f - 0.22f;
    constexpr float lmid = -2.184424571137427f;  // log2(0.22)
    if (Y > 0.f && ill > 0.f) {
        const float lill = __log2f(ill);
        const float adj = ill <= mid ? mid * ex2_a(shadows * (lill - lmid))
                                     : rest * pow_e((ill - mid) * (1.f / rest), highlights) + mid;
        return detail == 1.f ? adj * __fdividef(Y, ill) : adj * ex2_a(detail * (lY - lill));
    }
    const float adj = ill <= mid ? mid * pow_e(ill / mid, shadows) : rest * pow_e((ill - mid) / rest, highlights) + mid;
    return adj * pow_e(Y / ill, detail);
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
    float freq = 1.f, amp = 1.f;
    float sum = noise2(P, G, px, py);
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        freq *= 0.5f;
        amp *= 0.5f;
        sum += noise2(P, G, px * freq, py * freq) * amp;
    }
    return sum * (1.f / 1.875f);  // norm = 1 + 1/2 + 1/4 + 1/8
}

// toneCurve (demosaic.metal:607-609): sigmoid(powr(0.95 x, 0.5)), rescaled
// so that 0 and 1 map to 0 and 1; powr(., 0.5) is the square root
// 0.5 (tanh(z) + 1) = 1 / (1 + e^(-2z))
__device__ __forceinline__ float tone_curve(float x, const SrgbArgs& a) {
    constexpr float k = -2.f * 1.4426950408889634f;  // -2 log2(e)
    const float z = a.slope * sqrt_a(0.95f * x) - 0.3f * a.slope;
    const float sg = __fdividef(1.f, 1.f + ex2_a(k * z));
    return (sg - a.sig0) * a.sig_rrange;
}

template <class S, class O>
__device__ __forceinline__ void post_pixel(const Plane<S, 4>& in, const Plane<S, 2>& grad, const PostStats& st,
                                           const int* P, const float2* G, const SrgbArgs& a, Plane<O, 4>& out,
                                           int x, int y) {
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
        const float lY = Y > 0.f ? __log2f(Y) : 0.f, rY = __fdividef(1.f, Y);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float2 abk = band_ab(a.band[k], x, y);
            const float ill = abk.x * Y + abk.y;
            float d = a.detail[k];
            if (d > 1.f) {
                float dd = (1.f - sstep_r(0.75f, kR_075_095, ill)) * sstep_r(0.05f, kR_005_010, ill);
                if (k == 2) {
                    const f2 g = ld2<S>(grad.px(x, y));
                    const float gl = sqrt_a(g.x * g.x + g.y * g.y);
                    const float sigma = sqrt_a(a.nlf[0] + a.nlf[1] * ill);
                    const float r6 = __fdividef(1.f, 6.f * sigma), r96 = __fdividef(1.f, 96.f * sigma);
                    dd = sstep_r(2.f * sigma, r6, gl) * (1.f - sstep_r(32.f * sigma, r96, gl)) * dd;
                }
                d = 1.f + (d - 1.f) * dd;
            }
            mask *= ltm_multiplier_y(Y, lY, ill, st.shadows, k == 0 ? st.highlights : 1.f, d) * rY;
        }
    }
    // ---- convertTosRGB
    const float black = st.black, white = 1.f;
    float brightening = 1.f;
    if (st.mean > 0.22f) brightening *= 0.22f / st.mean;
    const float gain = brightening / (white - black) * a.bias_mul;
    float pv[3];
#pragma unroll
    for (int c = 0; c < 3; c++) pv[c] = fmaxf(rin[c] - black, 0.f) * gain;
    if (a.saturation != 1.f) {
        const float luma = 0.2126f * pv[0] + 0.7152f * pv[1] + 0.0722f * pv[2];
#pragma unroll
        for (int c = 0; c < 3; c++)
            pv[c] = mixf(luma, pv[c], mixf(a.saturation, 1.f, sstep_r(0.75f, kR_075_200, pv[c])));
    }
    if (a.contrast != 1.f) {
#pragma unroll
        for (int c = 0; c < 3; c++) pv[c] = mixf(0.2f, pv[c], mixf(a.contrast, 1.f, sstep_r(0.9f, kR_090_200, pv[c])));
    }
    float rgb[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
        rgb[c] = fmaxf(a.rgb_cam[3 * c] * pv[0] + a.rgb_cam[3 * c + 1] * pv[1] + a.rgb_cam[3 * c + 2] * pv[2], 0.f);
    float sigma = 0.f;
    const bool lv = a.luma_var[0] != 0.f || a.luma_var[1] != 0.f;
    if (a.ltm) {
        if (mask > 1.f) {
            const float luma = 0.2126f * rgb[0] + 0.7152f * rgb[1] + 0.0722f * rgb[2];
            const float t = fminf(sqrt_a(luma), 1.f), s = sstep_r(0.5f, kR_050_080, luma);
            const float q = __fdividef(1.f - mask * luma, 1.f - luma);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float lifted = 1.f - (1.f - rgb[c]) * q;
                rgb[c] = mixf(rgb[c] * mask, mixf(lifted, rgb[c] * mask, s), t);
            }
        } else if (mask < 1.f) {
#pragma unroll
            for (int c = 0; c < 3; c++) rgb[c] *= mask;
        }
        if (lv) sigma = sqrt_a(a.luma_var[0] + a.luma_var[1] * mask * rin[1]);
    } else if (lv) {
        sigma = sqrt_a(a.luma_var[0] + a.luma_var[1] * rin[1]);
    }
    if (sigma > 0.f) {
        const float n = octave_noise(P, G, 0.5f * float(x), 0.5f * float(y));
#pragma unroll
        for (int c = 0; c < 3; c++) rgb[c] += sigma * n;
    }
    f4 o;
    float* ov = &o.x;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float v = tone_curve(fmaxf(rgb[c], 0.f), a);
        if (a.blacks > 0.f) v = (v - a.blacks) / (1.f - a.blacks);
        ov[c] = clampf(v, 0.f, 1.f);
    }
    o.w = 1.f;
    st4<O>(out.px(x, y), o);
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
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= in.w) return;
    const PostStats st = *st_;
    const int y0 = blockIdx.y * (blockDim.y * PS_ROWS) + threadIdx.y;
#pragma unroll 1
    for (int r = 0; r < PS_ROWS; r++) {
        const int y = y0 + r * blockDim.y;
        if (y < in.h) post_pixel<S, O>(in, grad, st, P, G, a, out, x, y);
    }
}

}  // namespace

size_t post_ab_bytes(int w, int h) {
    return (size_t(w >> 4) * (h >> 4) + size_t(w >> 2) * (h >> 2) + size_t(w) * h) * sizeof(float2);
}

template <class S, class O>
int launch_post(const PostArgs<S>& pa, Plane<O, 4> out, cudaStream_t s) {
    const dim3 b(32, 8);
    auto grid = [&](int w, int h) { return dim3((w + 31) / 32, (h + 7) / 8); };
    int launches = 0;
    if (pa.denoise) {
        k_hist<S><<<grid(pa.den[3].w, pa.den[3].h), b, 0, s>>>(pa.den[3], pa.hist);
        launches++;
    }
    k_post_tables<<<1, 256, 0, s>>>(pa.hist, uint32_t(pa.den[3].w) * uint32_t(pa.den[3].h), pa.denoise ? 0 : 1,
                                   pa.stats, pa.raw, pa.perm, pa.grad_tab);
    launches++;
    SrgbArgs a{};
    const gls_demosaic_params& p = *pa.params;
    std::memcpy(a.m, pa.y2c, sizeof(a.m));
    std::memcpy(a.rgb_cam, p.rgb_cam, sizeof(a.rgb_cam));
    a.contrast = p.rgb_conversion.contrast;
    a.saturation = p.rgb_conversion.saturation;
    a.slope = p.rgb_conversion.tone_curve_slope;
    {  // the tone curve's end points, sigmoid(x, s) = 0.5 (tanh(s x - 0.3 s) + 1) (demosaic.metal:600-602)
        const float sl = a.slope;
        const float s0 = 0.5f * (std::tanh(sl * 0.f - 0.3f * sl) + 1.f);
        const float s1 = 0.5f * (std::tanh(sl * 1.f - 0.3f * sl) + 1.f);
        a.sig0 = s0;
        a.sig_rrange = 1.f / (s1 - s0);
    }
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
        GuideBands<S> gb;
        float2* ab = pa.ab;
        gb.first[0] = 0;
        for (int k = 0; k < 3; k++) {
            const Plane<S, 4>& g = pa.den[lv[k]];
            gb.guide[k] = g;
            gb.out[k] = ab;
            gb.tiles_x[k] = (g.w + GB_TX - 1) / GB_TX;
            gb.first[k + 1] = gb.first[k] + gb.tiles_x[k] * ((g.h + GB_OY - 1) / GB_OY);
            a.band[k] = {ab, g.w, g.h, float(g.w) / float(in.w), float(g.h) / float(in.h),
                         (g.w == in.w && g.h == in.h) ? 1 : 0};
            ab += size_t(g.w) * g.h;
        }
        k_guided_box<S><<<gb.first[3], dim3(GB_TX, GB_TY), 0, s>>>(gb, p.ltm.eps);
        launches++;
    }
    k_post_srgb<S, O><<<dim3((in.w + 31) / 32, (in.h + 8 * PS_ROWS - 1) / (8 * PS_ROWS)), b, 0, s>>>(
        in, pa.grad2, pa.stats, pa.perm,
                                                       reinterpret_cast<const float2*>(pa.grad_tab), a, out);
    return launches + 1;
}

template int launch_post<float, float>(const PostArgs<float>&, Plane<float, 4>, cudaStream_t);
template int launch_post<float, __half>(const PostArgs<float>&, Plane<__half, 4>, cudaStream_t);
template int launch_post<__half, float>(const PostArgs<__half>&, Plane<float, 4>, cudaStream_t);
template int launch_post<__half, __half>(const PostArgs<__half>&, Plane<__half, 4>, cudaStream_t);

}  // namespace gls
