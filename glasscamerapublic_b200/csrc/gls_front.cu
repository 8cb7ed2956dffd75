// gls_front.cu — front-end kernels of the raw path: Bayer unpack + scale,
// Sobel + noise-adaptive gradient blur, the high-noise quad-domain raw
// denoise, the fused three-pass demosaic with highlight blend and colour
// transform, and the luma/chroma despeckle.
//
// Each kernel is a shared-memory halo tile: a block loads its tile plus the
// stencil's halo once (clamped to the image edge), computes every
// intermediate plane of the stencil chain for the tile in shared memory and
// writes only the final plane. Intermediate planes of the reference
// (Sobel image, green image, red/blue temporary) never reach HBM.
#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

// --------------------------------------------------------------------------
// scaleRawData, demosaic.metal:96-118. One thread per 2 horizontal pixels.
// value = max(ls * k_c * (raw - black) + 0.1, 0), k_c = scale_mul[c]*0.9/65535
// (formed on the host in double). The black-level subtraction is integer;
// the FP32 operations are explicitly rounded (no contraction) so the FP32
// plane is bit-identical to the CPU oracle's FP32 run.
template <class S>
__global__ void __launch_bounds__(256) k_scale_raw(const uint16_t* __restrict__ raw, size_t raw_pitch,
                                                   Plane<S, 1> out, ScaleArgs a) {
    const int x2 = (blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const int y = blockIdx.y;
    if (x2 >= out.w || y >= out.h) return;
    const ushort2 rv = *reinterpret_cast<const ushort2*>(raw + size_t(y) * raw_pitch + x2);
    float ls = 1.f;
    if (a.lsc > 0.f) {
        const float dx = __fsub_rn(float(x2), a.cx), dy = __fsub_rn(float(y & ~1), a.cy);
        const float r = __fdiv_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))), a.clen);
        ls = __fadd_rn(1.f, __fmul_rn(__fmul_rn(a.lsc, r), r));
    }
    float v[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int c = bayer_channel(a.pattern, x2 + i, y);
        const int d = int(i == 0 ? rv.x : rv.y) - a.black;
        const float k = a.lsc > 0.f ? __fmul_rn(ls, a.k[c]) : a.k[c];
        v[i] = fmaxf(__fadd_rn(a.lsc > 0.f ? __fmul_rn(k, float(d)) : __fmul_rn(float(d), k), 0.1f), 0.f);
    }
    S* o = out.px(x2, y);
    if constexpr (is_half<S>::value) {
        *reinterpret_cast<__half2*>(o) = __floats2half2_rn(v[0], v[1]);
    } else {
        *reinterpret_cast<float2*>(o) = make_float2(v[0], v[1]);
    }
}

// The same for 8 pixels per thread, with 16-byte raw loads (rows 16-byte
// aligned, width a multiple of 8): the per-pixel arithmetic is the one
// above, so the planes are identical.
template <class S>
__global__ void __launch_bounds__(256) k_scale_raw8(const uint16_t* __restrict__ raw, size_t raw_pitch,
                                                    Plane<S, 1> out, ScaleArgs a) {
    const int x8 = (blockIdx.x * blockDim.x + threadIdx.x) * 8;
    const int y = blockIdx.y;
    if (x8 >= out.w || y >= out.h) return;
    const uint4 rv = *reinterpret_cast<const uint4*>(raw + size_t(y) * raw_pitch + x8);
    const uint32_t rw[4] = {rv.x, rv.y, rv.z, rv.w};
    float ls[8];
#pragma unroll
    for (int j = 0; j < 4; j++) {  // lens shading per pixel pair, as the 2-pixel kernel forms it
        float l = 1.f;
        if (a.lsc > 0.f) {
            const float dx = __fsub_rn(float(x8 + 2 * j), a.cx), dy = __fsub_rn(float(y & ~1), a.cy);
            const float r = __fdiv_rn(__fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy))), a.clen);
            l = __fadd_rn(1.f, __fmul_rn(__fmul_rn(a.lsc, r), r));
        }
        ls[2 * j] = ls[2 * j + 1] = l;
    }
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int c = bayer_channel(a.pattern, x8 + i, y);
        const int d = int((rw[i >> 1] >> (16 * (i & 1))) & 0xffffu) - a.black;
        const float k = a.lsc > 0.f ? __fmul_rn(ls[i], a.k[c]) : a.k[c];
        v[i] = fmaxf(__fadd_rn(a.lsc > 0.f ? __fmul_rn(k, float(d)) : __fmul_rn(float(d), k), 0.1f), 0.f);
    }
    S* o = out.px(x8, y);
    if constexpr (is_half<S>::value) {
        uint4 u;
        __half2 h0 = __floats2half2_rn(v[0], v[1]), h1 = __floats2half2_rn(v[2], v[3]);
        __half2 h2 = __floats2half2_rn(v[4], v[5]), h3 = __floats2half2_rn(v[6], v[7]);
        u.x = *reinterpret_cast<uint32_t*>(&h0);
        u.y = *reinterpret_cast<uint32_t*>(&h1);
        u.z = *reinterpret_cast<uint32_t*>(&h2);
        u.w = *reinterpret_cast<uint32_t*>(&h3);
        *reinterpret_cast<uint4*>(o) = u;
    } else {
        reinterpret_cast<float4*>(o)[0] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float4*>(o)[1] = make_float4(v[4], v[5], v[6], v[7]);
    }
}

// --------------------------------------------------------------------------
// rawImageSobel + sampledConvolutionSobel fused, demosaic.metal:120-213.
// Output tile 32 x 32 per 256-thread block. Shared memory: the scaled raw
// tile with a 5-pixel halo (+1 right/bottom for the bilinear pair) and the
// Sobel (gx, gy) tile with a 4/5-pixel halo. The blur taps are bilinear
// samples at integer + fractional offsets (host-computed Gaussian folding).
constexpr int SB_TW = 32, SB_TH = 32;
constexpr int SB_RW = SB_TW + 11, SB_RH = SB_TH + 11;  // raw tile, origin -5
constexpr int SB_SW = SB_TW + 9, SB_SH = SB_TH + 9;    // sobel tile, origin -4

template <class S>
__global__ void __launch_bounds__(256) k_sobel_blur(Plane<S, 1> raw, Plane<S, 2> out, BlurArgs a) {
    __shared__ float sraw[SB_RH][SB_RW];
    __shared__ float2 ssob[SB_SH][SB_SW];
    const int x0 = blockIdx.x * SB_TW, y0 = blockIdx.y * SB_TH;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nth = blockDim.x * blockDim.y;
    for (int i = tid; i < SB_RW * SB_RH; i += nth) {
        const int ty = i / SB_RW, tx = i % SB_RW;
        sraw[ty][tx] = to_f(*raw.pxc(x0 - 5 + tx, y0 - 5 + ty));
    }
    __syncthreads();
    const float inv = a.inv_sqrt45;
    for (int i = tid; i < SB_SW * SB_SH; i += nth) {
        const int ty = i / SB_SW, tx = i % SB_SW;
        // Sobel at the clamped position of this tile entry
        const int qx = clampi(x0 - 4 + tx, 0, raw.w - 1) - (x0 - 5);
        const int qy = clampi(y0 - 4 + ty, 0, raw.h - 1) - (y0 - 5);
        const float tl = sraw[qy - 1][qx - 1], tc = sraw[qy - 1][qx], tr = sraw[qy - 1][qx + 1];
        const float ml = sraw[qy][qx - 1], mr = sraw[qy][qx + 1];
        const float bl = sraw[qy + 1][qx - 1], bc = sraw[qy + 1][qx], br = sraw[qy + 1][qx + 1];
        const float gx = ((tl - tr) + 2.f * (ml - mr) + (bl - br)) * inv;
        const float gy = ((tl - bl) + 2.f * (tc - bc) + (tr - br)) * inv;
        ssob[ty][tx] = make_float2(gx, gy);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < SB_TH; r += blockDim.y) {
        const int x = x0 + threadIdx.x, y = y0 + r;
        if (x >= out.w || y >= out.h) continue;
        const int lx = threadIdx.x + 4, ly = r + 4;  // sobel tile index of (x, y)
        auto conv = [&](int first, int n, float res[4]) {
            float s0 = 0, s1 = 0, s2 = 0, s3 = 0, norm = 0;
            for (int t = first; t < first + n; t++) {
                const float w = a.w[t];
                const int ix = lx + a.ix[t], iy = ly + a.iy[t];
                const float ax = a.fx[t], ay = a.fy[t];
                const float2 p00 = ssob[iy][ix], p01 = ssob[iy][ix + 1];
                const float2 p10 = ssob[iy + 1][ix], p11 = ssob[iy + 1][ix + 1];
                auto bil = [&](float v00, float v01, float v10, float v11) {
                    const float top = v00 + (v01 - v00) * ax;
                    const float bot = v10 + (v11 - v10) * ax;
                    return top + (bot - top) * ay;
                };
                s0 += w * bil(p00.x, p01.x, p10.x, p11.x);
                s1 += w * bil(p00.y, p01.y, p10.y, p11.y);
                s2 += w * bil(fabsf(p00.x), fabsf(p01.x), fabsf(p10.x), fabsf(p11.x));
                s3 += w * bil(fabsf(p00.y), fabsf(p01.y), fabsf(p10.y), fabsf(p11.y));
                norm += w;
            }
            res[0] = s0 / norm;
            res[1] = s1 / norm;
            res[2] = s2 / norm;
            res[3] = s3 / norm;
        };
        float res[4];
        conv(0, a.n1, res);
        const float sigma = sqrtf(a.var0 + a.var1 * sraw[r + 5][threadIdx.x + 5]);
        if (sqrtf(res[0] * res[0] + res[1] * res[1]) < 4.f * sigma) conv(a.n1, a.n2, res);
        st2<S>(out.px(x, y), f2{copysignf(res[2], res[0]), copysignf(res[3], res[1])});
    }
}

// The FP16-storage path's form of the same stencil. The wide blur's 25
// bilinear taps sit on a 5 x 5 grid whose x offsets depend on the column
// only and y offsets on the row only, and whose weights are the Gaussian's
// 2 x 2 block sums, a product of a row and a column factor: the blur is
// separable. It runs as a horizontal pass (5 taps, two texels each) into
// shared memory and a vertical pass over it, a third of the operations of
// the 25 bilinear taps. The one tap off the grid is the corner, which the
// folding puts at (width/2, width/2) = (4.5, 4.5) (demosaic_utils.cpp:984)
// instead of (4, 4): it is moved there by one correction term. The factors
// come from the tap table (row and column sums of the weights), so the
// result is the 25-tap blur up to FP32 rounding of the factorisation.
struct SepSmem {
    float sraw[SB_RH][SB_RW];
    float2 ssob[SB_SH][SB_SW];
    float4 hsum[SB_SH][SB_TW];  // horizontal pass: (gx, gy, |gx|, |gy|) per sobel-tile row, output column
    float u[5], v[5];
    int ix[5], iy[5];
    float fx[5], fy[5];
    float total, wc, cdx, cdy;  // corner tap: weight, offset
};

__device__ __forceinline__ float4 bil4(const float2 (*ssob)[SB_SW], int ix, int iy, float ax, float ay) {
    const float2 p00 = ssob[iy][ix], p01 = ssob[iy][ix + 1];
    const float2 p10 = ssob[iy + 1][ix], p11 = ssob[iy + 1][ix + 1];
    auto bil = [&](float v00, float v01, float v10, float v11) {
        const float top = v00 + (v01 - v00) * ax;
        const float bot = v10 + (v11 - v10) * ax;
        return top + (bot - top) * ay;
    };
    return make_float4(bil(p00.x, p01.x, p10.x, p11.x), bil(p00.y, p01.y, p10.y, p11.y),
                       bil(fabsf(p00.x), fabsf(p01.x), fabsf(p10.x), fabsf(p11.x)),
                       bil(fabsf(p00.y), fabsf(p01.y), fabsf(p10.y), fabsf(p11.y)));
}

template <class S>
__global__ void __launch_bounds__(256) k_sobel_blur_sep(Plane<S, 1> raw, Plane<S, 2> out, BlurArgs a) {
    __shared__ SepSmem sm;
    const int x0 = blockIdx.x * SB_TW, y0 = blockIdx.y * SB_TH;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nth = blockDim.x * blockDim.y;
    if (tid == 0) {  // the wide taps' grid: row / column offsets and weight factors
        const int b = a.n1;
        float total = 0.f, rs[5] = {0, 0, 0, 0, 0}, cs[5] = {0, 0, 0, 0, 0};
        for (int r = 0; r < 5; r++)
            for (int c = 0; c < 5; c++) {
                const float w = a.w[b + r * 5 + c];
                rs[r] += w;
                cs[c] += w;
                total += w;
            }
        for (int k = 0; k < 5; k++) {
            sm.u[k] = rs[k] / total;  // u_r v_c = W_rc for a separable table
            sm.v[k] = cs[k];
            sm.ix[k] = a.ix[b + k];
            sm.fx[k] = a.fx[b + k];
            sm.iy[k] = a.iy[b + k * 5];
            sm.fy[k] = a.fy[b + k * 5];
        }
        sm.total = total;
        sm.wc = a.w[b + 24];
        sm.cdx = float(a.ix[b + 24]) + a.fx[b + 24];
        sm.cdy = float(a.iy[b + 24]) + a.fy[b + 24];
    }
    for (int i = tid; i < SB_RW * SB_RH; i += nth) {
        const int ty = i / SB_RW, tx = i % SB_RW;
        sm.sraw[ty][tx] = to_f(*raw.pxc(x0 - 5 + tx, y0 - 5 + ty));
    }
    __syncthreads();
    const float inv = a.inv_sqrt45;
    for (int i = tid; i < SB_SW * SB_SH; i += nth) {
        const int ty = i / SB_SW, tx = i % SB_SW;
        const int qx = clampi(x0 - 4 + tx, 0, raw.w - 1) - (x0 - 5);
        const int qy = clampi(y0 - 4 + ty, 0, raw.h - 1) - (y0 - 5);
        const float tl = sm.sraw[qy - 1][qx - 1], tc = sm.sraw[qy - 1][qx], tr = sm.sraw[qy - 1][qx + 1];
        const float ml = sm.sraw[qy][qx - 1], mr = sm.sraw[qy][qx + 1];
        const float bl = sm.sraw[qy + 1][qx - 1], bc = sm.sraw[qy + 1][qx], br = sm.sraw[qy + 1][qx + 1];
        const float gx = ((tl - tr) + 2.f * (ml - mr) + (bl - br)) * inv;
        const float gy = ((tl - bl) + 2.f * (tc - bc) + (tr - br)) * inv;
        sm.ssob[ty][tx] = make_float2(gx, gy);
    }
    __syncthreads();
    // horizontal pass: every sobel-tile row, every output column
    for (int i = tid; i < SB_SH * SB_TW; i += nth) {
        const int ry = i / SB_TW, cx = i % SB_TW;
        float4 h = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int c = 0; c < 5; c++) {
            const int xx = cx + 4 + sm.ix[c];
            const float ax = sm.fx[c], vc = sm.v[c];
            const float2 p0 = sm.ssob[ry][xx], p1 = sm.ssob[ry][xx + 1];
            h.x += vc * (p0.x + (p1.x - p0.x) * ax);
            h.y += vc * (p0.y + (p1.y - p0.y) * ax);
            h.z += vc * (fabsf(p0.x) + (fabsf(p1.x) - fabsf(p0.x)) * ax);
            h.w += vc * (fabsf(p0.y) + (fabsf(p1.y) - fabsf(p0.y)) * ax);
        }
        sm.hsum[ry][cx] = h;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < SB_TH; r += blockDim.y) {
        const int x = x0 + threadIdx.x, y = y0 + r;
        if (x >= out.w || y >= out.h) continue;
        const int lx = threadIdx.x + 4, ly = r + 4;  // sobel tile index of (x, y)
        float res[4];
        {  // narrow blur: its few taps directly
            float s0 = 0, s1 = 0, s2 = 0, s3 = 0, norm = 0;
            for (int t = 0; t < a.n1; t++) {
                const float w = a.w[t];
                const float4 b = bil4(sm.ssob, lx + a.ix[t], ly + a.iy[t], a.fx[t], a.fy[t]);
                s0 += w * b.x;
                s1 += w * b.y;
                s2 += w * b.z;
                s3 += w * b.w;
                norm += w;
            }
            res[0] = s0 / norm;
            res[1] = s1 / norm;
            res[2] = s2 / norm;
            res[3] = s3 / norm;
        }
        const float sigma = sqrtf(a.var0 + a.var1 * sm.sraw[r + 5][threadIdx.x + 5]);
        if (sqrtf(res[0] * res[0] + res[1] * res[1]) < 4.f * sigma) {
            // vertical pass over the horizontal sums, then the corner tap moved
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const int yy = ly + sm.iy[k];
                const float ay = sm.fy[k], ur = sm.u[k];
                const float4 h0 = sm.hsum[yy][threadIdx.x], h1 = sm.hsum[yy + 1][threadIdx.x];
                acc.x += ur * (h0.x + (h1.x - h0.x) * ay);
                acc.y += ur * (h0.y + (h1.y - h0.y) * ay);
                acc.z += ur * (h0.z + (h1.z - h0.z) * ay);
                acc.w += ur * (h0.w + (h1.w - h0.w) * ay);
            }
            const float gxo = float(sm.ix[4]) + sm.fx[4], gyo = float(sm.iy[4]) + sm.fy[4];  // the grid corner
            const float4 on = bil4(sm.ssob, lx + int(floorf(gxo)), ly + int(floorf(gyo)), gxo - floorf(gxo),
                                   gyo - floorf(gyo));
            const float4 at = bil4(sm.ssob, lx + int(floorf(sm.cdx)), ly + int(floorf(sm.cdy)),
                                   sm.cdx - floorf(sm.cdx), sm.cdy - floorf(sm.cdy));
            const float it = 1.f / sm.total;
            res[0] = (acc.x + sm.wc * (at.x - on.x)) * it;
            res[1] = (acc.y + sm.wc * (at.y - on.y)) * it;
            res[2] = (acc.z + sm.wc * (at.z - on.z)) * it;
            res[3] = (acc.w + sm.wc * (at.w - on.w)) * it;
        }
        st2<S>(out.px(x, y), f2{copysignf(res[2], res[0]), copysignf(res[3], res[1])});
    }
}

// --------------------------------------------------------------------------
// High-noise raw branch, raw_converter.cpp:195-202: bayerToRawRGBA ->
// despeckleRawRGBAImage -> crossDenoiseRawRGBAImage -> rawRGBAToBayer.
// The quad gather/scatter is folded into the two stencil kernels.

// despeckle_3x3x4 on the quad image read straight from the Bayer plane,
// demosaic.metal:1025-1092. Output: quad RGBA plane.
template <class S>
__global__ void __launch_bounds__(256) k_raw_despeckle(Plane<S, 1> bayer, Plane<S, 2> grad, Plane<S, 4> quad,
                                                       RawDenoiseArgs a) {
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= quad.w || qy >= quad.h) return;
    const f2 g = ld2<S>(grad.px(2 * qx, 2 * qy));
    const float gradient = sqrtf(g.x * g.x + g.y * g.y);
    float res[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int ox = kBayer[a.pattern][c][0], oy = kBayer[a.pattern][c][1];
        float fmx = 0, smx = 0, fmn = 65504.f, smn = 65504.f;
#pragma unroll
        for (int i = -1; i <= 1; i++)
#pragma unroll
            for (int j = -1; j <= 1; j++) {
                const int sx = clampi(qx + i, 0, quad.w - 1), sy = clampi(qy + j, 0, quad.h - 1);
                const float v = to_f(*bayer.px(2 * sx + ox, 2 * sy + oy));
                smx = v >= fmx ? fmx : fmaxf(v, smx);
                fmx = fmaxf(v, fmx);
                smn = v <= fmn ? fmn : fminf(v, smn);
                fmn = fminf(v, fmn);
            }
        const float s = to_f(*bayer.px(2 * qx + ox, 2 * qy + oy));
        const float sigma = sqrtf(a.var[c] * s);
        const float tex = 1.f - 0.5f * smoothstepf(1.f, 2.f, gradient / sigma);
        const float mn = mixf(fmn, smn, tex * (1.f - smoothstepf(2.f * sigma, 8.f * sigma, smn - fmn)));
        const float mx = mixf(fmx, smx, tex * (1.f - smoothstepf(sigma, 4.f * sigma, fmx - smx)));
        res[c] = clampf(s, mn, mx);
    }
    st4<S>(quad.px(qx, qy), f4{res[0], res[1], res[2], res[3]});
}

// crossDenoiseRawRGBAImage, demosaic.metal:999-1023, writing the result
// back into the Bayer plane (rawRGBAToBayer, :980-997).
template <class S>
__global__ void __launch_bounds__(256) k_raw_cross_denoise(Plane<S, 4> quad, Plane<S, 1> bayer, RawDenoiseArgs a) {
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= quad.w || qy >= quad.h) return;
    const f4 p = ld4<S>(quad.px(qx, qy));
    const float pc[4] = {p.x, p.y, p.z, p.w};
    float inv[4];
#pragma unroll
    for (int c = 0; c < 4; c++) inv[c] = 1.f / (a.strength * sqrtf(a.var[c] * (pc[c] + 0.0001f)));
    float sum[4] = {0, 0, 0, 0}, sw = 0;
    if (is_half<S>::value && a.fast) {
        // FP16 storage: the weight exp(-2 d^2) as exp2(-|(p - s) k|^2) with
        // k = inv sqrt(2 log2 e) folded into the inverse, and (p - s) k as
        // one FMA per channel with p k precomputed
        float ki[4], pk[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            ki[c] = inv[c] * 1.6986436f;  // sqrt(2 log2 e)
            pk[c] = pc[c] * ki[c];
        }
#pragma unroll
        for (int j = -2; j <= 2; j++)
#pragma unroll
            for (int i = -2; i <= 2; i++) {
                const f4 s = ld4<S>(quad.pxc(qx + i, qy + j));
                const float sc[4] = {s.x, s.y, s.z, s.w};
                float d2 = 0.f;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float d = fmaf(-sc[c], ki[c], pk[c]);
                    d2 = fmaf(d, d, d2);
                }
                float w;
                asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(w) : "f"(-d2));
#pragma unroll
                for (int c = 0; c < 4; c++) sum[c] = fmaf(w, sc[c], sum[c]);
                sw += w;
            }
    } else {
        for (int j = -2; j <= 2; j++)
            for (int i = -2; i <= 2; i++) {
                const f4 s = ld4<S>(quad.pxc(qx + i, qy + j));
                const float sc[4] = {s.x, s.y, s.z, s.w};
                float d2 = 0;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float d = (pc[c] - sc[c]) * inv[c];
                    d2 += d * d;
                }
                const float w = a.fast ? __expf(-2.f * d2) : expf(-2.f * d2);
#pragma unroll
                for (int c = 0; c < 4; c++) sum[c] += w * sc[c];
                sw += w;
            }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int ox = kBayer[a.pattern][c][0], oy = kBayer[a.pattern][c][1];
        *bayer.px(2 * qx + ox, 2 * qy + oy) = from_f<S>(sum[c] / sw);
    }
}

// --------------------------------------------------------------------------
// Fused demosaic: interpolateGreen (demosaic.metal:215-316) ->
// interpolateRedBlue (:318-416) -> interpolateRedBlueAtGreen (:418-521) ->
// blendHighlightsImage (:523-564) -> optional transformImage (:649-662).
// Output tile 32 x 32; halos: red/blue temporary +-3, green +-5, raw +-7.
constexpr int DM_TW = 32, DM_TH = 32;
constexpr int DM_RW = DM_TW + 14, DM_RH = DM_TH + 14;  // raw, origin -7
constexpr int DM_GW = DM_TW + 10, DM_GH = DM_TH + 10;  // green + gradient, origin -5
constexpr int DM_CW = DM_TW + 6, DM_CH = DM_TH + 6;    // red/blue temporary, origin -3

struct DemosaicSmem {
    float raw[DM_RH][DM_RW];
    float green[DM_GH][DM_GW];
    float2 grad[DM_GH][DM_GW];
    float tmp[3][DM_CH][DM_CW];
};


// The three interpolation passes evaluate the reference's formulas at two
// kinds of site: the Bayer sites of the pass's own colour copy a value, the
// others run the full stencil. Within a Bayer row the two kinds alternate,
// so a lane takes a horizontal pair of sites (one of each) and no warp
// runs both branches. Tiles whose staged region reaches past the image
// edge (clamped, repeated positions) take the sites one by one instead.
// The per-site arithmetic is the same in both orders.
struct DmSites {
    int rx, ry, bx, by;
    __device__ __forceinline__ bool red(int px, int py) const { return (rx & 1) == (px & 1) && (ry & 1) == (py & 1); }
    __device__ __forceinline__ bool blue(int px, int py) const { return (bx & 1) == (px & 1) && (by & 1) == (py & 1); }
};

// interpolateGreen (demosaic.metal:215-316) at raw-tile index (lx, ly) of a
// red or blue site; gg = |gradient| there.
__device__ __forceinline__ float dm_green(const DemosaicSmem& sm, int lx, int ly, float2 gg, const DemosaicArgs& a,
                                          float lowNoise) {
    const float kPi = 3.14159265358979323846f;
    auto R = [&](int di, int dj) { return sm.raw[ly + dj][lx + di]; };
    const float gl = R(-1, 0), gr = R(1, 0), gu = R(0, -1), gd = R(0, 1);
    const float cxy = R(0, 0);
    const float cl = R(-2, 0), cr = R(2, 0), cu = R(0, -2), cd = R(0, 2);
    const float c2ave = (R(-1, -1) + R(1, -1) + R(-1, 1) + R(1, 1)) / 4.f;
    const float gave = (gl + gr + gu + gd) / 4.f;
    const float glfx = (gl + gr) / 2.f, glfy = (gu + gd) / 2.f;
    const float ghfx = ((cl + cr) - 2.f * cxy) / 4.f, ghfy = ((cu + cd) - 2.f * cxy) / 4.f;
    const float sd = sqrtf(a.gv0 + a.gv1 * gave);
    const float glen = sqrtf(gg.x * gg.x + gg.y * gg.y);
    const float gthr = smoothstepf(sd, 4.f * sd, glen);
    const float lowthr = 1.f - smoothstepf(2.f * sd, 8.f * sd, glen);
    const float sharp = (0.5f + 0.5f * lowNoise) * gthr * (1.f + lowNoise * lowthr);
    const float hl = 1.f - smoothstepf(0.25f, 1.f, fmaxf(cxy, fmaxf(fmaxf(cl, cr), fmaxf(cu, cd))));
    float dir = 2.f * atan2f(gg.y, gg.x) / kPi;
    if (a.gv1 < 1e-3f) {
        dir = dir < 0.5f ? mixf(dir, 0.f, 1.f - smoothstepf(0.3f, 0.45f, dir))
                         : mixf(dir, 1.f, smoothstepf(1.f - 0.45f, 1.f - 0.3f, dir));
    }
    const float cmin = fminf(cxy, fminf(gave, c2ave)), cmax = fmaxf(cxy, fmaxf(gave, c2ave));
    const float white = cmin / cmax;
    const float k = hl * white * sharp;
    const float gex = glfx - k * ghfx, gey = glfy - k * ghfy;
    float g = mixf(gey, gex, dir);
    const float maxo = mixf(1.f, 1.5f, white), mino = mixf(1.f, 0.5f, white);
    const float gmax = fmaxf(fmaxf(gl, gr), fmaxf(gu, gd));
    const float gmin = fminf(fminf(gl, gr), fminf(gu, gd));
    return clampf(g, mino * gmin, maxo * gmax);
}

// interpolateRedBlue (demosaic.metal:318-416) at a red or blue site: the
// other colour; green-tile index (gx, gy), raw-tile index (lx, ly).
__device__ __forceinline__ float dm_redblue(const DemosaicSmem& sm, int gx, int gy, int lx, int ly, bool red,
                                            const DemosaicArgs& a) {
    const float kPi = 3.14159265358979323846f;
    auto R = [&](int di, int dj) { return sm.raw[ly + dj][lx + di]; };
    auto G = [&](int di, int dj) { return sm.green[gy + dj][gx + di]; };
    const float g0 = G(0, 0), c1 = R(0, 0);
    const float c2tl = R(-1, -1), c2tr = R(1, -1), c2bl = R(-1, 1), c2br = R(1, 1);
    const float c2ave = (c2tl + c2tr + c2bl + c2br) / 4.f;
    const float gctl = G(-1, -1) - c2tl, gctr = G(1, -1) - c2tr, gcbl = G(-1, 1) - c2bl, gcbr = G(1, 1) - c2br;
    const float gtl2 = G(-2, -2), gtr2 = G(2, -2), gbl2 = G(-2, 2), gbr2 = G(2, 2);
    const float gctl2 = gtl2 - R(-2, -2), gctr2 = gtr2 - R(2, -2), gcbl2 = gbl2 - R(-2, 2), gcbr2 = gbr2 - R(2, 2);
    const float v0 = red ? a.rv0 : a.bv0, v1 = red ? a.rv1 : a.bv1;
    const float sd = sqrtf(v0 + v1 * c2ave);
    const float2 gg = sm.grad[gy][gx];
    const float dir = 1.f - 2.f * atan2f(gg.y, gg.x) / kPi;
    const float gthr = smoothstepf(sd, 4.f * sd, sqrtf(gg.x * gg.x + gg.y * gg.y));
    const float alpha = mixf(0.5f, dir, gthr);
    const float hl = 1.f - smoothstepf(0.25f, 1.f, fmaxf(g0, fmaxf(fmaxf(gtr2, gbl2), fmaxf(gtl2, gbr2))));
    const float gc = g0 - c1;
    const float aa = (gctr + gcbl) / 2.f + hl * (gctr2 + gcbl2 - 2.f * gc) / 8.f;
    const float bb = (gctl + gcbr) / 2.f + hl * (gctl2 + gcbr2 - 2.f * gc) / 8.f;
    const float c2 = g0 - mixf(aa, bb, alpha);
    const float c2max = fmaxf(fmaxf(c2tl, c2tr), fmaxf(c2bl, c2br));
    const float c2min = fminf(fminf(c2tl, c2tr), fminf(c2bl, c2br));
    return clampf(c2, c2min, c2max);
}

// interpolateRedBlueAtGreen (demosaic.metal:418-521) at a green site:
// tmp-tile index (cx, cy), green-tile index of the gradient (gx, gy).
__device__ __forceinline__ void dm_rb_at_green(const DemosaicSmem& sm, int cx, int cy, float2 gg, const DemosaicArgs& a,
                                               float rgb[3]) {
    const float kPi = 3.14159265358979323846f;
    auto P = [&](int di, int dj, int c) { return sm.tmp[c][cy + dj][cx + di]; };
    const float g0 = P(0, 0, 1);
    const float lr = P(-1, 0, 0), lg = P(-1, 0, 1), lb = P(-1, 0, 2);
    const float rr = P(1, 0, 0), rg = P(1, 0, 1), rb = P(1, 0, 2);
    const float ur = P(0, -1, 0), ug = P(0, -1, 1), ub = P(0, -1, 2);
    const float dr = P(0, 1, 0), dg = P(0, 1, 1), db = P(0, 1, 2);
    const float red_ave = (lr + rr + ur + dr) / 4.f, blue_ave = (lb + rb + ub + db) / 4.f;
    const float grl = lg - lr, grr = rg - rr, gru = ug - ur, grd = dg - dr;
    const float gbl = lg - lb, gbr = rg - rb, gbu = ug - ub, gbd = dg - db;
    const float grl3 = P(-3, 0, 1) - P(-3, 0, 0), grr3 = P(3, 0, 1) - P(3, 0, 0);
    const float gru3 = P(0, -3, 1) - P(0, -3, 0), grd3 = P(0, 3, 1) - P(0, 3, 0);
    const float gbl3 = P(-3, 0, 1) - P(-3, 0, 2), gbr3 = P(3, 0, 1) - P(3, 0, 2);
    const float gbu3 = P(0, -3, 1) - P(0, -3, 2), gbd3 = P(0, 3, 1) - P(0, 3, 2);
    const float dir = 2.f * atan2f(gg.y, gg.x) / kPi;
    const float glen = sqrtf(gg.x * gg.x + gg.y * gg.y);
    const float rsd = sqrtf(a.rv0 + a.rv1 * red_ave), bsd = sqrtf(a.bv0 + a.bv1 * blue_ave);
    const float ralpha = mixf(0.5f, dir, smoothstepf(rsd, 4.f * rsd, glen));
    const float balpha = mixf(0.5f, dir, smoothstepf(bsd, 4.f * bsd, glen));
    const float hl = 1.f - smoothstepf(0.25f, 1.f, fmaxf(g0, fmaxf(fmaxf(rg, lg), fmaxf(dg, ug))));
    const float red_v = g0 - mixf((gru + grd) / 2.f - hl * ((grd3 - gru) - (grd - gru3)) / 8.f,
                                  (grl + grr) / 2.f - hl * ((grr3 - grl) - (grr - grl3)) / 8.f, ralpha);
    const float blue_v = g0 - mixf((gbu + gbd) / 2.f - hl * ((gbd3 - gbu) - (gbd - gbu3)) / 8.f,
                                   (gbl + gbr) / 2.f - hl * ((gbr3 - gbl) - (gbr - gbl3)) / 8.f, balpha);
    rgb[0] = clampf(red_v, fminf(fminf(lr, rr), fminf(ur, dr)), fmaxf(fmaxf(lr, rr), fmaxf(ur, dr)));
    rgb[1] = g0;
    rgb[2] = clampf(blue_v, fminf(fminf(lb, rb), fminf(ub, db)), fmaxf(fmaxf(lb, rb), fmaxf(ub, db)));
}

// blendHighlightsImage (clip = 1) and the optional colour transform.
__device__ __forceinline__ f4 dm_finish(float rgb[3], const DemosaicArgs& a) {
    const float clip = 1.f;
    if (rgb[0] > clip || rgb[1] > clip || rgb[2] > clip) {
        const float s3 = 1.7320508f;
        const float c0[3] = {rgb[0], rgb[1], rgb[2]};
        const float c1[3] = {fminf(rgb[0], clip), fminf(rgb[1], clip), fminf(rgb[2], clip)};
        const float l0x = c0[0] + c0[1] + c0[2], l0y = s3 * c0[0] - s3 * c0[1], l0z = -c0[0] - c0[1] + 2.f * c0[2];
        const float l1y = s3 * c1[0] - s3 * c1[1], l1z = -c1[0] - c1[1] + 2.f * c1[2];
        const float sum0 = l0y * l0y + l0z * l0z, sum1 = l1y * l1y + l1z * l1z;
        const float chr = sum0 > 0.f ? sqrtf(sum1 / sum0) : 1.f;
        const float ly = l0y * chr, lz = l0z * chr;
        rgb[0] = (l0x + (s3 / 2.f) * ly - 0.5f * lz) / 3.f;
        rgb[1] = (l0x - (s3 / 2.f) * ly - 0.5f * lz) / 3.f;
        rgb[2] = (l0x + lz) / 3.f;
    }
    f4 o;
    if (a.transform) {
        o.x = a.m[0] * rgb[0] + a.m[1] * rgb[1] + a.m[2] * rgb[2];
        o.y = a.m[3] * rgb[0] + a.m[4] * rgb[1] + a.m[5] * rgb[2];
        o.z = a.m[6] * rgb[0] + a.m[7] * rgb[1] + a.m[8] * rgb[2];
    } else {
        o.x = rgb[0]; o.y = rgb[1]; o.z = rgb[2];
    }
    o.w = 0.f;
    return o;
}

template <class S>
__global__ void __launch_bounds__(256) k_demosaic(Plane<S, 1> raw, Plane<S, 2> grad, Plane<S, 4> out, DemosaicArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DemosaicSmem& sm = *reinterpret_cast<DemosaicSmem*>(smem_raw);
    const int x0 = blockIdx.x * DM_TW, y0 = blockIdx.y * DM_TH;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nth = blockDim.x * blockDim.y;
    const int W = raw.w, H = raw.h;
    const DmSites st{kBayer[a.pattern][0][0], kBayer[a.pattern][0][1], kBayer[a.pattern][2][0], kBayer[a.pattern][2][1]};
    // the staged region (raw tile, origin -7) lies inside the image: positions
    // are not clamped, and sites alternate along every row
    const bool inner = x0 >= 7 && y0 >= 7 && x0 + DM_RW - 7 <= W && y0 + DM_RH - 7 <= H;
    // a site (px, py) is red or blue iff the parity of px ^ py is this
    const int rb_par = (st.rx ^ st.ry) & 1;

    for (int i = tid; i < DM_RW * DM_RH; i += nth) {
        const int ty = i / DM_RW, tx = i % DM_RW;
        sm.raw[ty][tx] = to_f(*raw.pxc(x0 - 7 + tx, y0 - 7 + ty));
    }
    for (int i = tid; i < DM_GW * DM_GH; i += nth) {
        const int ty = i / DM_GW, tx = i % DM_GW;
        const f2 g = ld2<S>(grad.pxc(x0 - 5 + tx, y0 - 5 + ty));
        sm.grad[ty][tx] = make_float2(fabsf(g.x), fabsf(g.y));
    }
    __syncthreads();

    // ---- green at the clamped position of every green-tile entry
    const float lowNoise = 1.f - smoothstepf(3.5e-4f, 2e-3f, a.gv1);
    if (inner) {
        // entry pairs (2k, 2k + 1) of a row: one red/blue site, one green site
        for (int i = tid; i < (DM_GW / 2) * DM_GH; i += nth) {
            const int ty = i / (DM_GW / 2), tx0 = 2 * (i % (DM_GW / 2));
            const int py = y0 - 5 + ty;
            const int trb = tx0 + (((x0 - 5 + tx0) ^ py ^ rb_par) & 1);  // the pair's red/blue entry
            const int tg = tx0 + tx0 + 1 - trb;
            sm.green[ty][tg] = sm.raw[ty + 2][tg + 2];
            sm.green[ty][trb] = dm_green(sm, trb + 2, ty + 2, sm.grad[ty][trb], a, lowNoise);
        }
    } else {
        for (int i = tid; i < DM_GW * DM_GH; i += nth) {
            const int ty = i / DM_GW, tx = i % DM_GW;
            const int px = clampi(x0 - 5 + tx, 0, W - 1), py = clampi(y0 - 5 + ty, 0, H - 1);
            const int lx = px - (x0 - 7), ly = py - (y0 - 7);  // raw-tile index of the clamped position
            sm.green[ty][tx] = (st.red(px, py) || st.blue(px, py)) ? dm_green(sm, lx, ly, sm.grad[ty][tx], a, lowNoise)
                                                                   : sm.raw[ly][lx];
        }
    }
    __syncthreads();

    // ---- red/blue temporary at the clamped position of every tmp-tile entry
    if (inner) {
        for (int i = tid; i < (DM_CW / 2) * DM_CH; i += nth) {
            const int ty = i / (DM_CW / 2), tx0 = 2 * (i % (DM_CW / 2));
            const int px0 = x0 - 3 + tx0, py = y0 - 3 + ty;
            const int trb = tx0 + ((px0 ^ py ^ rb_par) & 1);
            const int tg = tx0 + tx0 + 1 - trb;
            const int prb = x0 - 3 + trb;
            const bool red = st.red(prb, py);
            sm.tmp[0][ty][tg] = 0.f;
            sm.tmp[1][ty][tg] = sm.green[ty + 2][tg + 2];
            sm.tmp[2][ty][tg] = 0.f;
            const float c2 = dm_redblue(sm, trb + 2, ty + 2, trb + 4, ty + 4, red, a);
            const float c1 = sm.raw[ty + 4][trb + 4];
            sm.tmp[0][ty][trb] = red ? c1 : c2;
            sm.tmp[1][ty][trb] = sm.green[ty + 2][trb + 2];
            sm.tmp[2][ty][trb] = red ? c2 : c1;
        }
    } else {
        for (int i = tid; i < DM_CW * DM_CH; i += nth) {
            const int ty = i / DM_CW, tx = i % DM_CW;
            const int px = clampi(x0 - 3 + tx, 0, W - 1), py = clampi(y0 - 3 + ty, 0, H - 1);
            const int gx = px - (x0 - 5), gy = py - (y0 - 5);  // green-tile index
            const int lx = px - (x0 - 7), ly = py - (y0 - 7);  // raw-tile index
            const bool red = st.red(px, py), blue = st.blue(px, py);
            float o0, o1, o2;
            if (!(red || blue)) {
                o0 = 0.f;
                o1 = sm.green[gy][gx];
                o2 = 0.f;
            } else {
                const float c2 = dm_redblue(sm, gx, gy, lx, ly, red, a);
                const float c1 = sm.raw[ly][lx];
                o0 = red ? c1 : c2;
                o1 = sm.green[gy][gx];
                o2 = red ? c2 : c1;
            }
            sm.tmp[0][ty][tx] = o0;
            sm.tmp[1][ty][tx] = o1;
            sm.tmp[2][ty][tx] = o2;
        }
    }
    __syncthreads();

    // ---- red/blue at green sites, highlights, colour transform: a lane
    //      takes the pixel pair (2k, 2k + 1) of a tile row
    for (int i = tid; i < (DM_TW / 2) * DM_TH; i += nth) {
        const int r = i / (DM_TW / 2), c0 = 2 * (i % (DM_TW / 2));
        const int y = y0 + r;
        if (y >= H) continue;
#pragma unroll
        for (int e = 0; e < 2; e++) {
            // the pair's green site first, so both lanes of a warp branch alike
            const int cg = c0 + (((x0 + c0) ^ y ^ rb_par ^ 1) & 1);
            const int c = e == 0 ? cg : c0 + c0 + 1 - cg;
            const int x = x0 + c;
            if (x >= W) continue;
            const int cx = c + 3, cy = r + 3;  // tmp-tile index of (x, y)
            float rgb[3];
            if (st.red(x, y) || st.blue(x, y)) {
                rgb[0] = sm.tmp[0][cy][cx];
                rgb[1] = sm.tmp[1][cy][cx];
                rgb[2] = sm.tmp[2][cy][cx];
            } else {
                dm_rb_at_green(sm, cx, cy, sm.grad[r + 5][c + 5], a, rgb);
            }
            st4<S>(out.px(x, y), dm_finish(rgb, a));
        }
    }
}

// --------------------------------------------------------------------------
// despeckleLumaMedianChromaImage, demosaic.metal:1161-1283.
// The chroma pair (Cb, Cr) of a pixel as one value for the median
// network: a half2 on the FP16 path (the planes hold halves, so packing is
// exact and one min/max instruction serves both channels), two floats on the
// FP32 path.
template <class S>
struct ChromaPair {
    float2 v;
    __device__ __forceinline__ static ChromaPair of(const f4& p) { return {make_float2(p.y, p.z)}; }
    __device__ __forceinline__ static ChromaPair mn(ChromaPair a, ChromaPair b) {
        return {make_float2(fminf(a.v.x, b.v.x), fminf(a.v.y, b.v.y))};
    }
    __device__ __forceinline__ static ChromaPair mx(ChromaPair a, ChromaPair b) {
        return {make_float2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y))};
    }
    __device__ __forceinline__ float2 get() const { return v; }
};
template <>
struct ChromaPair<__half> {
    __half2 v;
    __device__ __forceinline__ static ChromaPair of(const f4& p) { return {__floats2half2_rn(p.y, p.z)}; }
    __device__ __forceinline__ static ChromaPair mn(ChromaPair a, ChromaPair b) { return {__hmin2(a.v, b.v)}; }
    __device__ __forceinline__ static ChromaPair mx(ChromaPair a, ChromaPair b) { return {__hmax2(a.v, b.v)}; }
    __device__ __forceinline__ float2 get() const { return __half22float2(v); }
};

// a row of three sorted: (lo, mid, hi)
template <class C>
struct Sorted3 {
    C lo, mid, hi;
};
template <class C>
__device__ __forceinline__ Sorted3<C> sort3(C a, C b, C c) {
    const C l1 = C::mn(a, b), h1 = C::mx(a, b);   // a, b ordered
    const C m2 = C::mn(h1, c), hi = C::mx(h1, c);  // the largest
    return {C::mn(l1, m2), C::mx(l1, m2), hi};
}
template <class C>
__device__ __forceinline__ C med3(C a, C b, C c) {
    return C::mx(C::mn(a, b), C::mn(C::mx(a, b), c));
}
// The median of a 3 x 3 neighbourhood from its three sorted rows: the median
// of (the largest row minimum, the median of the row medians, the smallest
// row maximum). Exact (the median is one of the nine values), as the
// reference's min/max elimination network (demosaic.metal:1161-1196) is;
// the adjoint's selection network (gls_front_jvp.cu) picks the same value.
template <class C>
__device__ __forceinline__ C median9_rows(const Sorted3<C>& r0, const Sorted3<C>& r1, const Sorted3<C>& r2) {
    const C lo = C::mx(C::mx(r0.lo, r1.lo), r2.lo);
    const C hi = C::mn(C::mn(r0.hi, r1.hi), r2.hi);
    return med3(lo, med3(r0.mid, r1.mid, r2.mid), hi);
}

// The luma part of one output pixel from its 3 x 3 neighbourhood, rows
// r0..r2 of 3 loaded pixels each, taken in the reference's order
// (j = -1..1, i = -1..1).
__device__ __forceinline__ float despeckle_luma(const f4 (&r0)[3], const f4 (&r1)[3], const f4 (&r2)[3], float va,
                                                float vb) {
    float fmx = 0.f, smx = 0.f, fmn = INFINITY, smn = INFINITY, sample = 0.f;
    const f4* rows[3] = {r0, r1, r2};
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float v = rows[j][i].x;
            smx = (v <= fmx && v > smx) ? v : smx;
            smx = v > fmx ? fmx : smx;
            fmx = v > fmx ? v : fmx;
            smn = (v >= fmn && v < smn) ? v : smn;
            smn = v < fmn ? fmn : smn;
            fmn = v < fmn ? v : fmn;
            if (i == 1 && j == 1) sample = v;
        }
    const float sigma = sqrtf(va + vb * sample);
    const float mn = mixf(smn, fmn, smoothstepf(sigma, 4.f * sigma, smn - fmn));
    const float mx = mixf(smx, fmx, smoothstepf(sigma, 4.f * sigma, fmx - smx));
    return clampf(sample, mn, mx);
}

// Two vertically adjacent pixels per thread: they share two of their three
// neighbourhood rows (12 loads instead of 18), and the chroma medians share
// the sorting of those rows (four row sorts for two medians).
template <class S>
__global__ void __launch_bounds__(256) k_despeckle(Plane<S, 4> in, Plane<S, 4> out, float va, float vb) {
    using C = ChromaPair<S>;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = 2 * (blockIdx.y * blockDim.y + threadIdx.y);
    if (x >= in.w || y >= in.h) return;
    f4 r[4][3];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) r[j][i] = ld4<S>(in.pxc(x + i - 1, y + j - 1));
    Sorted3<C> rs[4];
#pragma unroll
    for (int j = 0; j < 4; j++) rs[j] = sort3(C::of(r[j][0]), C::of(r[j][1]), C::of(r[j][2]));
    const float2 m0 = median9_rows(rs[0], rs[1], rs[2]).get();
    st4<S>(out.px(x, y), f4{despeckle_luma(r[0], r[1], r[2], va, vb), m0.x, m0.y, 0.f});
    if (y + 1 < in.h) {
        const float2 m1 = median9_rows(rs[1], rs[2], rs[3]).get();
        st4<S>(out.px(x, y + 1), f4{despeckle_luma(r[1], r[2], r[3], va, vb), m1.x, m1.y, 0.f});
    }
}

// transformImage, demosaic.metal:649-662, from plane S4 to an output of
// element type O (float or half), w = 0.
template <class S, class O>
__global__ void __launch_bounds__(256) k_transform(Plane<S, 4> in, Plane<O, 4> out, Mat3Args m) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= in.w || y >= in.h) return;
    const f4 p = ld4<S>(in.px(x, y));
    f4 o;
    o.x = m.m[0] * p.x + m.m[1] * p.y + m.m[2] * p.z;
    o.y = m.m[3] * p.x + m.m[4] * p.y + m.m[5] * p.z;
    o.z = m.m[6] * p.x + m.m[7] * p.y + m.m[8] * p.z;
    o.w = 0.f;
    st4<O>(out.px(x, y), o);
}

// plain copy with element conversion (for output views)
template <class S, class O>
__global__ void __launch_bounds__(256) k_convert4(Plane<S, 4> in, Plane<O, 4> out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= in.w || y >= in.h) return;
    st4<O>(out.px(x, y), ld4<S>(in.px(x, y)));
}

// ------------------------------------------------------------------ launchers
static inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

template <class S>
void launch_scale_raw(const uint16_t* raw, size_t raw_pitch, Plane<S, 1> out, const ScaleArgs& a, cudaStream_t s) {
    const bool wide = (uintptr_t(raw) % 16) == 0 && (raw_pitch % 8) == 0 && (out.w % 8) == 0 &&
                      (uintptr_t(out.p) % 16) == 0 && (out.pitch % 8) == 0;
    if (wide) {
        dim3 b(128, 1);
        dim3 g((out.w / 8 + b.x - 1) / b.x, out.h);
        k_scale_raw8<S><<<g, b, 0, s>>>(raw, raw_pitch, out, a);
        return;
    }
    dim3 b(128, 1);
    dim3 g((out.w / 2 + b.x - 1) / b.x, out.h);
    k_scale_raw<S><<<g, b, 0, s>>>(raw, raw_pitch, out, a);
}

template <class S>
void launch_sobel_blur(Plane<S, 1> raw, Plane<S, 2> out, const BlurArgs& a, cudaStream_t s) {
    dim3 b(32, 8);
    dim3 g((raw.w + SB_TW - 1) / SB_TW, (raw.h + SB_TH - 1) / SB_TH);
    // the FP16-storage path takes the separable form of the 5 x 5 wide blur;
    // the FP32 plain path evaluates the reference's 25 bilinear taps
    if (is_half<S>::value && a.n2 == 25) k_sobel_blur_sep<S><<<g, b, 0, s>>>(raw, out, a);
    else k_sobel_blur<S><<<g, b, 0, s>>>(raw, out, a);
}

template <class S>
void launch_raw_denoise(Plane<S, 1> bayer, Plane<S, 2> grad, Plane<S, 4> quad, const RawDenoiseArgs& a,
                        cudaStream_t s) {
    dim3 b(32, 8);
    k_raw_despeckle<S><<<grid2(quad.w, quad.h, b), b, 0, s>>>(bayer, grad, quad, a);
    k_raw_cross_denoise<S><<<grid2(quad.w, quad.h, b), b, 0, s>>>(quad, bayer, a);
}

template <class S>
void launch_demosaic(Plane<S, 1> raw, Plane<S, 2> grad, Plane<S, 4> out, const DemosaicArgs& a, cudaStream_t s) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_demosaic<S>), int(sizeof(DemosaicSmem)));
    dim3 b(32, 8);
    dim3 g((raw.w + DM_TW - 1) / DM_TW, (raw.h + DM_TH - 1) / DM_TH);
    k_demosaic<S><<<g, b, sizeof(DemosaicSmem), s>>>(raw, grad, out, a);
}

template <class S>
void launch_despeckle(Plane<S, 4> in, Plane<S, 4> out, float va, float vb, cudaStream_t s) {
    dim3 b(32, 8);
    k_despeckle<S><<<grid2(in.w, (in.h + 1) / 2, b), b, 0, s>>>(in, out, va, vb);
}

template <class S, class O>
void launch_transform(Plane<S, 4> in, Plane<O, 4> out, const Mat3Args& m, cudaStream_t s) {
    dim3 b(32, 8);
    k_transform<S, O><<<grid2(in.w, in.h, b), b, 0, s>>>(in, out, m);
}

template <class S, class O>
void launch_convert4(Plane<S, 4> in, Plane<O, 4> out, cudaStream_t s) {
    dim3 b(32, 8);
    k_convert4<S, O><<<grid2(in.w, in.h, b), b, 0, s>>>(in, out);
}

#define GLS_INST(S)                                                                                            \
    template void launch_scale_raw<S>(const uint16_t*, size_t, Plane<S, 1>, const ScaleArgs&, cudaStream_t);  \
    template void launch_sobel_blur<S>(Plane<S, 1>, Plane<S, 2>, const BlurArgs&, cudaStream_t);              \
    template void launch_raw_denoise<S>(Plane<S, 1>, Plane<S, 2>, Plane<S, 4>, const RawDenoiseArgs&,         \
                                        cudaStream_t);                                                         \
    template void launch_demosaic<S>(Plane<S, 1>, Plane<S, 2>, Plane<S, 4>, const DemosaicArgs&, cudaStream_t); \
    template void launch_despeckle<S>(Plane<S, 4>, Plane<S, 4>, float, float, cudaStream_t);                  \
    template void launch_transform<S, float>(Plane<S, 4>, Plane<float, 4>, const Mat3Args&, cudaStream_t);    \
    template void launch_transform<S, __half>(Plane<S, 4>, Plane<__half, 4>, const Mat3Args&, cudaStream_t);  \
    template void launch_convert4<S, float>(Plane<S, 4>, Plane<float, 4>, cudaStream_t);                      \
    template void launch_convert4<S, __half>(Plane<S, 4>, Plane<__half, 4>, cudaStream_t);
GLS_INST(float)
GLS_INST(__half)
#undef GLS_INST

}  // namespace gls
