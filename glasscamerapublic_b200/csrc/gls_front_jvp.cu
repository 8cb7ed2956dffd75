// gls_front_jvp.cu — forward-mode derivatives of the raw front end with
// respect to the raw green noise model, for the adjoint's last two
// parameters:
//   theta30 moves raw_nlf.a[1] and a[3] together: the green variance offset
//           gv0 of the demosaic (getRawVariance, demosaic.hpp:186-193);
//   theta31 moves raw_nlf.b[1] and b[3] together: the green variance slope
//           gv1 of the demosaic and the G / G2 variances of the high-noise
//           raw branch (despeckleRawRGBAImage and crossDenoiseRawRGBAImage,
//           demosaic.metal:999-1092).
// The gradient plane depends on them only through the blur-radius switch of
// sampledConvolutionSobel (piecewise constant), so its tangent is zero.
//
// Every pass recomputes its forward pass (gls_front.cu) from the retained
// FP32 planes with dual numbers (value, d/dtheta30, d/dtheta31), one pixel
// per thread, neighbours read clamp-to-edge as the tiled forward reads them.
// Branches, clamps and order statistics are decided on the values, as the
// forward decides them. The last pass dots the despeckled image's tangents
// with dL/d(despeckled image) from the reverse sweep, per block, summed in
// block order on the host.
#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

namespace {

struct Dv {
    float v, a, b;  // value, d/dtheta30, d/dtheta31
};

__device__ __forceinline__ Dv dc(float v) { return {v, 0.f, 0.f}; }
__device__ __forceinline__ Dv operator+(Dv x, Dv y) { return {x.v + y.v, x.a + y.a, x.b + y.b}; }
__device__ __forceinline__ Dv operator-(Dv x, Dv y) { return {x.v - y.v, x.a - y.a, x.b - y.b}; }
__device__ __forceinline__ Dv operator-(Dv x) { return {-x.v, -x.a, -x.b}; }
__device__ __forceinline__ Dv operator*(Dv x, Dv y) { return {x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b}; }
__device__ __forceinline__ Dv operator/(Dv x, Dv y) {
    const float q = x.v / y.v;
    return {q, (x.a - q * y.a) / y.v, (x.b - q * y.b) / y.v};
}
__device__ __forceinline__ Dv operator+(float y, Dv x) { return {y + x.v, x.a, x.b}; }
__device__ __forceinline__ Dv operator-(float y, Dv x) { return {y - x.v, -x.a, -x.b}; }
__device__ __forceinline__ Dv operator*(Dv x, float y) { return {x.v * y, x.a * y, x.b * y}; }
__device__ __forceinline__ Dv operator*(float y, Dv x) { return {y * x.v, y * x.a, y * x.b}; }
__device__ __forceinline__ Dv operator/(Dv x, float y) { return {x.v / y, x.a / y, x.b / y}; }
__device__ __forceinline__ Dv dsqrt_(Dv x) {
    const float s = sqrtf(x.v);
    const float k = s > 0.f ? 0.5f / s : 0.f;
    return {s, k * x.a, k * x.b};
}
__device__ __forceinline__ Dv dexp_(Dv x) {
    const float e = expf(x.v);
    return {e, e * x.a, e * x.b};
}
__device__ __forceinline__ Dv dmin_(Dv x, Dv y) { return y.v < x.v ? y : x; }  // fminf: the smaller value
__device__ __forceinline__ Dv dmax_(Dv x, Dv y) { return y.v > x.v ? y : x; }
__device__ __forceinline__ Dv dclamp_(Dv x, Dv lo, Dv hi) { return dmin_(dmax_(x, lo), hi); }
__device__ __forceinline__ Dv dmix_(Dv a, Dv b, Dv t) { return a + (b - a) * t; }
__device__ __forceinline__ Dv dsmooth_(Dv e0, Dv e1, Dv x) {  // smoothstepf
    const Dv t = dclamp_((x - e0) / (e1 - e0), dc(0.f), dc(1.f));
    return t * t * (3.f - 2.f * t);
}

constexpr float kPiJ = 3.14159265358979323846f;

struct JvpPlanes {
    int w, h;
    const float* scaled;   // Bayer plane after the raw branch (forward)
    const float* scaled0;  // Bayer plane before it (forward, high-noise branch)
    const float* quad;     // despeckled quads (forward, high-noise branch)
    const float* grad;     // 2 ch
    float4* qtan;          // d(quad)/dtheta31 (theta30 does not reach the raw branch)
    float2* rtan;          // d(Bayer)/dtheta
    Dv* green;            // W x H
    Dv* tmp;              // W x H x 3
    Dv* ycc;              // W x H x 3, the demosaic output (YCbCr)
};

__device__ __forceinline__ int cl(int v, int n) { return min(max(v, 0), n - 1); }

// despeckleRawRGBAImage (demosaic.metal:1025-1092): the order statistics of
// the 3 x 3 same-channel neighbourhood do not depend on theta; the clamp
// thresholds do, through sigma = sqrt(var[c] * s)
__global__ void __launch_bounds__(256) k_jvp_raw_despeckle(JvpPlanes P, RawDenoiseArgs a) {
    const int qw = P.w / 2, qh = P.h / 2;
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= qw || qy >= qh) return;
    const float2 g = reinterpret_cast<const float2*>(P.grad)[size_t(2 * qy) * P.w + 2 * qx];
    const float gradient = sqrtf(g.x * g.x + g.y * g.y);
    float tan[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int ox = kBayer[a.pattern][c][0], oy = kBayer[a.pattern][c][1];
        float fmx = 0, smx = 0, fmn = 65504.f, smn = 65504.f;
        for (int i = -1; i <= 1; i++)
            for (int j = -1; j <= 1; j++) {
                const int sx = cl(qx + i, qw), sy = cl(qy + j, qh);
                const float v = P.scaled0[size_t(2 * sy + oy) * P.w + 2 * sx + ox];
                smx = v >= fmx ? fmx : fmaxf(v, smx);
                fmx = fmaxf(v, fmx);
                smn = v <= fmn ? fmn : fminf(v, smn);
                fmn = fminf(v, fmn);
            }
        const float sv = P.scaled0[size_t(2 * qy + oy) * P.w + 2 * qx + ox];
        const Dv var = {a.var[c], 0.f, (c == 1 || c == 3) ? 1.f : 0.f};
        const Dv sigma = dsqrt_(var * sv);
        const Dv tex = 1.f - 0.5f * dsmooth_(dc(1.f), dc(2.f), dc(gradient) / sigma);
        const Dv mn = dmix_(dc(fmn), dc(smn), tex * (1.f - dsmooth_(2.f * sigma, 8.f * sigma, dc(smn - fmn))));
        const Dv mx = dmix_(dc(fmx), dc(smx), tex * (1.f - dsmooth_(sigma, 4.f * sigma, dc(fmx - smx))));
        tan[c] = dclamp_(dc(sv), mn, mx).b;
    }
    P.qtan[size_t(qy) * qw + qx] = make_float4(tan[0], tan[1], tan[2], tan[3]);
}

// crossDenoiseRawRGBAImage with dual G / G2 variances and dual quads,
// written to the Bayer positions the forward writes (rawRGBAToBayer)
__global__ void __launch_bounds__(256) k_jvp_cross_denoise(JvpPlanes P, RawDenoiseArgs a) {
    const int qw = P.w / 2, qh = P.h / 2;
    const int qx = blockIdx.x * blockDim.x + threadIdx.x, qy = blockIdx.y * blockDim.y + threadIdx.y;
    if (qx >= qw || qy >= qh) return;
    auto quad = [&](int x, int y, Dv q[4]) {
        const size_t i = size_t(y) * qw + x;
        const float4 v = reinterpret_cast<const float4*>(P.quad)[i];
        const float4 t = P.qtan[i];
        q[0] = {v.x, 0.f, t.x};
        q[1] = {v.y, 0.f, t.y};
        q[2] = {v.z, 0.f, t.z};
        q[3] = {v.w, 0.f, t.w};
    };
    Dv pc[4];
    quad(qx, qy, pc);
    Dv inv[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const Dv var = {a.var[c], 0.f, (c == 1 || c == 3) ? 1.f : 0.f};
        inv[c] = dc(1.f) / (a.strength * dsqrt_(var * (pc[c] + dc(0.0001f))));
    }
    Dv sum[4] = {dc(0.f), dc(0.f), dc(0.f), dc(0.f)}, sw = dc(0.f);
    for (int j = -2; j <= 2; j++)
        for (int i = -2; i <= 2; i++) {
            Dv sc[4];
            quad(cl(qx + i, qw), cl(qy + j, qh), sc);
            Dv d2 = dc(0.f);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const Dv d = (pc[c] - sc[c]) * inv[c];
                d2 = d2 + d * d;
            }
            const Dv w = dexp_(-2.f * d2);
#pragma unroll
            for (int c = 0; c < 4; c++) sum[c] = sum[c] + w * sc[c];
            sw = sw + w;
        }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const Dv o = sum[c] / sw;
        const int ox = kBayer[a.pattern][c][0], oy = kBayer[a.pattern][c][1];
        P.rtan[size_t(2 * qy + oy) * P.w + 2 * qx + ox] = make_float2(o.a, o.b);
    }
}

struct Raw {
    const JvpPlanes& P;
    int x, y;
    __device__ Dv operator()(int di, int dj) const {
        const size_t i = size_t(cl(y + dj, P.h)) * P.w + cl(x + di, P.w);
        const float2 t = P.rtan[i];
        return {P.scaled[i], t.x, t.y};
    }
};

__device__ __forceinline__ float2 absgrad(const JvpPlanes& P, int x, int y) {
    const float2 g = reinterpret_cast<const float2*>(P.grad)[size_t(y) * P.w + x];
    return make_float2(fabsf(g.x), fabsf(g.y));
}

// interpolateGreen (demosaic.metal:215-316)
__global__ void __launch_bounds__(256) k_jvp_green(JvpPlanes P, DemosaicArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= P.w || y >= P.h) return;
    const int rx = kBayer[a.pattern][0][0], ry = kBayer[a.pattern][0][1];
    const int bx = kBayer[a.pattern][2][0], by = kBayer[a.pattern][2][1];
    const Raw R{P, x, y};
    const bool red = (rx & 1) == (x & 1) && (ry & 1) == (y & 1);
    const bool blue = (bx & 1) == (x & 1) && (by & 1) == (y & 1);
    const Dv gv0 = {a.gv0, 1.f, 0.f}, gv1 = {a.gv1, 0.f, 1.f};
    Dv g;
    if (!(red || blue)) {
        g = R(0, 0);
    } else {
        const Dv lowNoise = 1.f - dsmooth_(dc(3.5e-4f), dc(2e-3f), gv1);
        const Dv gl = R(-1, 0), gr = R(1, 0), gu = R(0, -1), gd = R(0, 1);
        const Dv cxy = R(0, 0);
        const Dv cL = R(-2, 0), cR = R(2, 0), cU = R(0, -2), cD = R(0, 2);
        const Dv c2ave = (R(-1, -1) + R(1, -1) + R(-1, 1) + R(1, 1)) / 4.f;
        const Dv gave = (gl + gr + gu + gd) / 4.f;
        const float2 gg = absgrad(P, x, y);
        const Dv glfx = (gl + gr) / 2.f, glfy = (gu + gd) / 2.f;
        const Dv ghfx = ((cL + cR) - 2.f * cxy) / 4.f, ghfy = ((cU + cD) - 2.f * cxy) / 4.f;
        const Dv sd = dsqrt_(gv0 + gv1 * gave);
        const Dv glen = dc(sqrtf(gg.x * gg.x + gg.y * gg.y));
        const Dv gthr = dsmooth_(sd, 4.f * sd, glen);
        const Dv lowthr = 1.f - dsmooth_(2.f * sd, 8.f * sd, glen);
        const Dv sharp = (0.5f + 0.5f * lowNoise) * gthr * (1.f + lowNoise * lowthr);
        const Dv hl = 1.f - dsmooth_(dc(0.25f), dc(1.f), dmax_(cxy, dmax_(dmax_(cL, cR), dmax_(cU, cD))));
        float dir = 2.f * atan2f(gg.y, gg.x) / kPiJ;
        if (a.gv1 < 1e-3f) {
            dir = dir < 0.5f ? mixf(dir, 0.f, 1.f - smoothstepf(0.3f, 0.45f, dir))
                             : mixf(dir, 1.f, smoothstepf(1.f - 0.45f, 1.f - 0.3f, dir));
        }
        const Dv cmin = dmin_(cxy, dmin_(gave, c2ave)), cmax = dmax_(cxy, dmax_(gave, c2ave));
        const Dv white = cmin / cmax;
        const Dv k = hl * white * sharp;
        const Dv gex = glfx - k * ghfx, gey = glfy - k * ghfy;
        g = dmix_(gey, gex, dc(dir));
        const Dv maxo = dmix_(dc(1.f), dc(1.5f), white), mino = dmix_(dc(1.f), dc(0.5f), white);
        const Dv gmax = dmax_(dmax_(gl, gr), dmax_(gu, gd));
        const Dv gmin = dmin_(dmin_(gl, gr), dmin_(gu, gd));
        g = dclamp_(g, mino * gmin, maxo * gmax);
    }
    P.green[size_t(y) * P.w + x] = g;
}

// interpolateRedBlue (demosaic.metal:318-416)
__global__ void __launch_bounds__(256) k_jvp_red_blue(JvpPlanes P, DemosaicArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= P.w || y >= P.h) return;
    const int rx = kBayer[a.pattern][0][0], ry = kBayer[a.pattern][0][1];
    const int bx = kBayer[a.pattern][2][0], by = kBayer[a.pattern][2][1];
    const bool red = (rx & 1) == (x & 1) && (ry & 1) == (y & 1);
    const bool blue = (bx & 1) == (x & 1) && (by & 1) == (y & 1);
    auto G = [&](int di, int dj) { return P.green[size_t(cl(y + dj, P.h)) * P.w + cl(x + di, P.w)]; };
    Dv o0, o1, o2;
    if (!(red || blue)) {
        o0 = dc(0.f);
        o1 = G(0, 0);
        o2 = dc(0.f);
    } else {
        const Raw R{P, x, y};
        const Dv g0 = G(0, 0), c1 = R(0, 0);
        const Dv c2tl = R(-1, -1), c2tr = R(1, -1), c2bl = R(-1, 1), c2br = R(1, 1);
        const Dv c2ave = (c2tl + c2tr + c2bl + c2br) / 4.f;
        const Dv gctl = G(-1, -1) - c2tl, gctr = G(1, -1) - c2tr, gcbl = G(-1, 1) - c2bl, gcbr = G(1, 1) - c2br;
        const Dv gtl2 = G(-2, -2), gtr2 = G(2, -2), gbl2 = G(-2, 2), gbr2 = G(2, 2);
        const Dv gctl2 = gtl2 - R(-2, -2), gctr2 = gtr2 - R(2, -2), gcbl2 = gbl2 - R(-2, 2), gcbr2 = gbr2 - R(2, 2);
        const float v0 = red ? a.rv0 : a.bv0, v1 = red ? a.rv1 : a.bv1;
        const Dv sd = dsqrt_(v0 + v1 * c2ave);
        const float2 gg = absgrad(P, x, y);
        const float dir = 1.f - 2.f * atan2f(gg.y, gg.x) / kPiJ;
        const Dv gthr = dsmooth_(sd, 4.f * sd, dc(sqrtf(gg.x * gg.x + gg.y * gg.y)));
        const Dv alpha = dmix_(dc(0.5f), dc(dir), gthr);
        const Dv hl = 1.f - dsmooth_(dc(0.25f), dc(1.f), dmax_(g0, dmax_(dmax_(gtr2, gbl2), dmax_(gtl2, gbr2))));
        const Dv gc = g0 - c1;
        const Dv aa = (gctr + gcbl) / 2.f + hl * (gctr2 + gcbl2 - 2.f * gc) / 8.f;
        const Dv bb = (gctl + gcbr) / 2.f + hl * (gctl2 + gcbr2 - 2.f * gc) / 8.f;
        Dv c2 = g0 - dmix_(aa, bb, alpha);
        const Dv c2max = dmax_(dmax_(c2tl, c2tr), dmax_(c2bl, c2br));
        const Dv c2min = dmin_(dmin_(c2tl, c2tr), dmin_(c2bl, c2br));
        c2 = dclamp_(c2, c2min, c2max);
        if (red) {
            o0 = c1; o1 = g0; o2 = c2;
        } else {
            o0 = c2; o1 = g0; o2 = c1;
        }
    }
    Dv* t = P.tmp + (size_t(y) * P.w + x) * 3;
    t[0] = o0;
    t[1] = o1;
    t[2] = o2;
}

// interpolateRedBlueAtGreen (demosaic.metal:418-521), blendHighlightsImage
// (:523-564) and transformImage to YCbCr (:649-662)
__global__ void __launch_bounds__(256) k_jvp_rb_at_green(JvpPlanes P, DemosaicArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= P.w || y >= P.h) return;
    const int rx = kBayer[a.pattern][0][0], ry = kBayer[a.pattern][0][1];
    const int bx = kBayer[a.pattern][2][0], by = kBayer[a.pattern][2][1];
    const bool red = (rx & 1) == (x & 1) && (ry & 1) == (y & 1);
    const bool blue = (bx & 1) == (x & 1) && (by & 1) == (y & 1);
    auto T = [&](int di, int dj, int c) { return P.tmp[(size_t(cl(y + dj, P.h)) * P.w + cl(x + di, P.w)) * 3 + c]; };
    Dv rgb[3];
    if (red || blue) {
        rgb[0] = T(0, 0, 0);
        rgb[1] = T(0, 0, 1);
        rgb[2] = T(0, 0, 2);
    } else {
        const Dv g0 = T(0, 0, 1);
        const Dv lr = T(-1, 0, 0), lg = T(-1, 0, 1), lb = T(-1, 0, 2);
        const Dv rr = T(1, 0, 0), rg = T(1, 0, 1), rb = T(1, 0, 2);
        const Dv ur = T(0, -1, 0), ug = T(0, -1, 1), ub = T(0, -1, 2);
        const Dv dr = T(0, 1, 0), dg = T(0, 1, 1), db = T(0, 1, 2);
        const Dv red_ave = (lr + rr + ur + dr) / 4.f, blue_ave = (lb + rb + ub + db) / 4.f;
        const Dv grl = lg - lr, grr = rg - rr, gru = ug - ur, grd = dg - dr;
        const Dv gbl = lg - lb, gbr = rg - rb, gbu = ug - ub, gbd = dg - db;
        const Dv grl3 = T(-3, 0, 1) - T(-3, 0, 0), grr3 = T(3, 0, 1) - T(3, 0, 0);
        const Dv gru3 = T(0, -3, 1) - T(0, -3, 0), grd3 = T(0, 3, 1) - T(0, 3, 0);
        const Dv gbl3 = T(-3, 0, 1) - T(-3, 0, 2), gbr3 = T(3, 0, 1) - T(3, 0, 2);
        const Dv gbu3 = T(0, -3, 1) - T(0, -3, 2), gbd3 = T(0, 3, 1) - T(0, 3, 2);
        const float2 gg = absgrad(P, x, y);
        const float dir = 2.f * atan2f(gg.y, gg.x) / kPiJ;
        const Dv glen = dc(sqrtf(gg.x * gg.x + gg.y * gg.y));
        const Dv rsd = dsqrt_(a.rv0 + a.rv1 * red_ave), bsd = dsqrt_(a.bv0 + a.bv1 * blue_ave);
        const Dv ralpha = dmix_(dc(0.5f), dc(dir), dsmooth_(rsd, 4.f * rsd, glen));
        const Dv balpha = dmix_(dc(0.5f), dc(dir), dsmooth_(bsd, 4.f * bsd, glen));
        const Dv hl = 1.f - dsmooth_(dc(0.25f), dc(1.f), dmax_(g0, dmax_(dmax_(rg, lg), dmax_(dg, ug))));
        const Dv red_v = g0 - dmix_((gru + grd) / 2.f - hl * ((grd3 - gru) - (grd - gru3)) / 8.f,
                                    (grl + grr) / 2.f - hl * ((grr3 - grl) - (grr - grl3)) / 8.f, ralpha);
        const Dv blue_v = g0 - dmix_((gbu + gbd) / 2.f - hl * ((gbd3 - gbu) - (gbd - gbu3)) / 8.f,
                                     (gbl + gbr) / 2.f - hl * ((gbr3 - gbl) - (gbr - gbl3)) / 8.f, balpha);
        rgb[0] = dclamp_(red_v, dmin_(dmin_(lr, rr), dmin_(ur, dr)), dmax_(dmax_(lr, rr), dmax_(ur, dr)));
        rgb[1] = g0;
        rgb[2] = dclamp_(blue_v, dmin_(dmin_(lb, rb), dmin_(ub, db)), dmax_(dmax_(lb, rb), dmax_(ub, db)));
    }
    const float clip = 1.f;
    if (rgb[0].v > clip || rgb[1].v > clip || rgb[2].v > clip) {
        const float s3 = 1.7320508f;
        const Dv c0[3] = {rgb[0], rgb[1], rgb[2]};
        const Dv c1[3] = {dmin_(rgb[0], dc(clip)), dmin_(rgb[1], dc(clip)), dmin_(rgb[2], dc(clip))};
        const Dv l0x = c0[0] + c0[1] + c0[2], l0y = s3 * c0[0] - s3 * c0[1], l0z = -c0[0] - c0[1] + 2.f * c0[2];
        const Dv l1y = s3 * c1[0] - s3 * c1[1], l1z = -c1[0] - c1[1] + 2.f * c1[2];
        const Dv sum0 = l0y * l0y + l0z * l0z, sum1 = l1y * l1y + l1z * l1z;
        const Dv chr = sum0.v > 0.f ? dsqrt_(sum1 / sum0) : dc(1.f);
        const Dv ly = l0y * chr, lz = l0z * chr;
        rgb[0] = (l0x + (s3 / 2.f) * ly - 0.5f * lz) / 3.f;
        rgb[1] = (l0x - (s3 / 2.f) * ly - 0.5f * lz) / 3.f;
        rgb[2] = (l0x + lz) / 3.f;
    }
    Dv* o = P.ycc + (size_t(y) * P.w + x) * 3;
    o[0] = a.m[0] * rgb[0] + a.m[1] * rgb[1] + a.m[2] * rgb[2];
    o[1] = a.m[3] * rgb[0] + a.m[4] * rgb[1] + a.m[5] * rgb[2];
    o[2] = a.m[6] * rgb[0] + a.m[7] * rgb[1] + a.m[8] * rgb[2];
}

__device__ __forceinline__ void dsort2(Dv& a, Dv& b) {
    const Dv t = dmin_(a, b);
    b = dmax_(a, b);
    a = t;
}
__device__ __forceinline__ Dv dmedian9(Dv v[9]) {  // the forward's selection network
    dsort2(v[1], v[2]); dsort2(v[4], v[5]); dsort2(v[7], v[8]);
    dsort2(v[0], v[1]); dsort2(v[3], v[4]); dsort2(v[6], v[7]);
    dsort2(v[1], v[2]); dsort2(v[4], v[5]); dsort2(v[7], v[8]);
    dsort2(v[0], v[3]); dsort2(v[5], v[8]); dsort2(v[4], v[7]);
    dsort2(v[3], v[6]); dsort2(v[1], v[4]); dsort2(v[2], v[5]);
    dsort2(v[4], v[7]); dsort2(v[4], v[2]); dsort2(v[6], v[4]);
    dsort2(v[4], v[2]);
    return v[4];
}

// despeckleLumaMedianChromaImage (demosaic.metal:1161-1283), then
// sum over pixels of <dL/d(despeckled), d(despeckled)/dtheta> per block
__global__ void __launch_bounds__(256) k_jvp_despeckle_dot(JvpPlanes P, float va, float vb, const float* g_ds,
                                                           float* part) {
    __shared__ float red[8][2];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    float sa = 0.f, sb = 0.f;
    if (x < P.w && y < P.h) {
        Dv cb[9], cr[9];
        Dv fmx = dc(0.f), smx = dc(0.f), fmn = dc(INFINITY), smn = dc(INFINITY), sample = dc(0.f);
        int k = 0;
        for (int j = -1; j <= 1; j++)
            for (int i = -1; i <= 1; i++, k++) {
                const Dv* p = P.ycc + (size_t(cl(y + j, P.h)) * P.w + cl(x + i, P.w)) * 3;
                const Dv v = p[0];
                smx = (v.v <= fmx.v && v.v > smx.v) ? v : smx;
                smx = v.v > fmx.v ? fmx : smx;
                fmx = v.v > fmx.v ? v : fmx;
                smn = (v.v >= fmn.v && v.v < smn.v) ? v : smn;
                smn = v.v < fmn.v ? fmn : smn;
                fmn = v.v < fmn.v ? v : fmn;
                if (i == 0 && j == 0) sample = v;
                cb[k] = p[1];
                cr[k] = p[2];
            }
        const Dv sigma = dsqrt_(va + vb * sample);
        const Dv mn = dmix_(smn, fmn, dsmooth_(sigma, 4.f * sigma, smn - fmn));
        const Dv mx = dmix_(smx, fmx, dsmooth_(sigma, 4.f * sigma, fmx - smx));
        const Dv o[3] = {dclamp_(sample, mn, mx), dmedian9(cb), dmedian9(cr)};
        const float* g = g_ds + (size_t(y) * P.w + x) * 3;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            sa += g[c] * o[c].a;
            sb += g[c] * o[c].b;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_down_sync(0xffffffffu, sa, o);
        sb += __shfl_down_sync(0xffffffffu, sb, o);
    }
    if ((tid & 31) == 0) {
        red[tid >> 5][0] = sa;
        red[tid >> 5][1] = sb;
    }
    __syncthreads();
    if (tid < 2) {
        float v = 0.f;
        for (int w = 0; w < 8; w++) v += red[w][tid];
        part[(size_t(blockIdx.y) * gridDim.x + blockIdx.x) * 2 + tid] = v;
    }
}

}  // namespace

// scratch: quad tangents (float4, 16-byte aligned first), Bayer tangents
// (float2), then the dual green, red/blue temporary and YCbCr planes
static size_t quad_tan_bytes(int w, int h) { return size_t(w / 2) * size_t(h / 2) * sizeof(float4); }

size_t front_jvp_scratch_bytes(int w, int h) {
    const size_t n = size_t(w) * h;
    return quad_tan_bytes(w, h) + n * sizeof(float2) + n * sizeof(Dv) * 7;
}

int front_jvp_blocks(int w, int h) { return ((w + 31) / 32) * ((h + 7) / 8); }

void launch_front_jvp(const FrontJvpArgs& f, cudaStream_t s) {
    const size_t n = size_t(f.w) * f.h;
    unsigned char* sc = static_cast<unsigned char*>(f.scratch);
    JvpPlanes P;
    P.w = f.w;
    P.h = f.h;
    P.scaled = f.scaled;
    P.scaled0 = f.scaled0;
    P.quad = f.quad;
    P.grad = f.grad;
    P.qtan = reinterpret_cast<float4*>(sc);
    P.rtan = reinterpret_cast<float2*>(sc + quad_tan_bytes(f.w, f.h));
    P.green = reinterpret_cast<Dv*>(sc + quad_tan_bytes(f.w, f.h) + n * sizeof(float2));
    P.tmp = P.green + n;
    P.ycc = P.tmp + 3 * n;
    const dim3 b(32, 8), g((f.w + 31) / 32, (f.h + 7) / 8);
    cudaMemsetAsync(P.rtan, 0, n * sizeof(float2), s);
    if (f.high_noise) {  // the raw branch: despeckle, then cross denoise into the Bayer plane
        const dim3 gq((f.w / 2 + 31) / 32, (f.h / 2 + 7) / 8);
        k_jvp_raw_despeckle<<<gq, b, 0, s>>>(P, f.raw);
        k_jvp_cross_denoise<<<gq, b, 0, s>>>(P, f.raw);
    }
    k_jvp_green<<<g, b, 0, s>>>(P, f.dm);
    k_jvp_red_blue<<<g, b, 0, s>>>(P, f.dm);
    k_jvp_rb_at_green<<<g, b, 0, s>>>(P, f.dm);
    k_jvp_despeckle_dot<<<g, b, 0, s>>>(P, f.despeckle_va, f.despeckle_vb, f.g_ds, f.part);
}

}  // namespace gls
