// gls_blockmatch.cu — blockMatchingDenoiseImage (demosaic.metal:806-884):
// 21 x 21 non-local means with a PCA-space patch distance for luma, a
// chroma distance for chroma and a fixed spatial Gaussian:
//   lw = exp(-2 (|p - q|_8 s)^2),   s = 1 / (luma_mult sigma_Y (1 + gb edge))
//   cw = exp(-2 (lw^2 + (dCb m1 / cb)^2 + (dCr m2 / cb)^2))
//   w  = gaussian(0.1 |(i, j)|) * (lw, cw, cw)
// accumulated in FP32; output (Y, Cb, Cr, sum of luma weights).
//
// Both kernels stage the tile's window region (halo 10) in shared memory
// and give each thread a column of vertically adjacent pixels, which share
// all but one of their window rows: one staged neighbour feeds several
// taps. The kernel for the FP32 plain path evaluates the formula directly
// with correctly rounded exponentials (parity with the oracle's FP32 run);
// the FP16-storage path's kernel is arranged for the fewest FMA-pipe and
// shared-memory operations per tap.
#include <cmath>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "gls_common.cuh"
#include "gls_kernels.h"
#include "gls_pyramid_dev.cuh"

namespace gls {

__device__ __forceinline__ __half2 u2h_(uint32_t u) { return *reinterpret_cast<__half2*>(&u); }

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Per-pixel constants shared by both kernels.
struct BmConst {
    float in_y, in_cb, in_cr;
    float s;       // luma distance scale
    float c1, c2;  // chroma scales (dm / chroma_boost)
};

template <class S>
__device__ __forceinline__ BmConst bm_const(const BlockMatchArgs& a, Plane<S, 2> grad, int w, int h, int px, int py,
                                            float y, float cb, float cr) {
    BmConst k;
    k.in_y = y;
    k.in_cb = cb;
    k.in_cr = cr;
    float ls = 1.f;
    if (a.lsc > 0.f) {  // lensShading, demosaic.metal:91-93, at the pixel
        const float cx = float(w / 2), cy = float(h / 2);
        const float dx = float(px) - cx, dy = float(py) - cy;
        const float rr = sqrtf(dx * dx + dy * dy) / sqrtf(cx * cx + cy * cy);
        ls = 1.f + a.lsc * rr * rr;
    }
    const float sig0 = sqrtf(a.var_a[0] + a.var_b[0] * ls * y);
    const float sig1 = sqrtf(a.var_a[1] + a.var_b[1] * ls * y);
    const float sig2 = sqrtf(a.var_a[2] + a.var_b[2] * ls * y);
    const float dm0 = 1.f / (a.tm[0] * sig0), dm1 = 1.f / (a.tm[1] * sig1), dm2 = 1.f / (a.tm[2] * sig2);
    const f2 g = ld2<S>(grad.px(px, py));
    const float mag = sqrtf(g.x * g.x + g.y * g.y);
    const float edge = smoothstepf(2.f, 16.f, a.gradient_threshold * mag / sig0);
    k.s = dm0 / (1.f + a.gradient_boost * edge);
    k.c1 = dm1 / a.chroma_boost;
    k.c2 = dm2 / a.chroma_boost;
    return k;
}

__device__ __forceinline__ float spatial_weight(int i, int j) {  // gaussian(0.1 |(i, j)|)
    const float d = 0.1f * sqrtf(float(i * i + j * j));
    return expf(-2.f * d * d);
}

// ============================================================ FP32 plain path
// Two vertically adjacent pixels per thread, tile 32 x 16, FP32 staging.
constexpr int BP_TX = 32, BP_TY = 8, BP_W = BP_TX + 20, BP_H = 2 * BP_TY + 20;

struct BmPlainSmem {
    float4 pca[BP_H * BP_W][2];
    float4 ycc[BP_H * BP_W];
    float spatial[21 * 21];
};

struct BmPlainPix {
    float4 p0, p1;
    float kl;              // -2 log2(e) s^2
    float c1, c2, o1, o2;  // sqrt(2 log2 e) c, times the centre chroma
};

template <bool UP, bool LO>
__device__ __forceinline__ void bmp_row(const BmPlainSmem& sm, int base, int r, const BmPlainPix& u,
                                        const BmPlainPix& l, float (&acc)[10]) {
    const float kLk = 2.f * 1.4426950408889634f;
#pragma unroll
    for (int i = 0; i < 21; i++) {
        const float4 q0 = sm.pca[base + i][0], q1 = sm.pca[base + i][1];
        const float4 y = sm.ycc[base + i];
        auto tap = [&](const BmPlainPix& p, int j, int o) {
            float d, d2;
            d = q0.x - p.p0.x; d2 = d * d;
            d = q0.y - p.p0.y; d2 = fmaf(d, d, d2);
            d = q0.z - p.p0.z; d2 = fmaf(d, d, d2);
            d = q0.w - p.p0.w; d2 = fmaf(d, d, d2);
            d = q1.x - p.p1.x; d2 = fmaf(d, d, d2);
            d = q1.y - p.p1.y; d2 = fmaf(d, d, d2);
            d = q1.z - p.p1.z; d2 = fmaf(d, d, d2);
            d = q1.w - p.p1.w; d2 = fmaf(d, d, d2);
            const float lw = exp2f(p.kl * d2);
            const float e1 = fmaf(p.c1, y.y, -p.o1), e2 = fmaf(p.c2, y.z, -p.o2);
            const float cw = exp2f(-fmaf(kLk * lw, lw, fmaf(e1, e1, e2 * e2)));
            const float sw = sm.spatial[j * 21 + i];
            const float wy = sw * lw, wc = sw * cw;
            acc[o + 0] = fmaf(wy, y.x, acc[o + 0]);
            acc[o + 1] = fmaf(wc, y.y, acc[o + 1]);
            acc[o + 2] = fmaf(wc, y.z, acc[o + 2]);
            acc[o + 3] += wy;
            acc[o + 4] += wc;
        };
        if (UP) tap(u, r, 0);
        if (LO) tap(l, r - 1, 5);
    }
}

template <class S>
__global__ void __launch_bounds__(256) k_block_match_plain(Plane<S, 4> img, Plane<S, 2> grad, Plane<S, 8> pca,
                                                           Plane<S, 4> out, BlockMatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BmPlainSmem& sm = *reinterpret_cast<BmPlainSmem*>(smem_raw);
    const int x0 = blockIdx.x * BP_TX, y0 = blockIdx.y * (2 * BP_TY);
    const int tid = threadIdx.y * BP_TX + threadIdx.x;
    for (int k = tid; k < 441; k += 256) sm.spatial[k] = spatial_weight(k % 21 - 10, k / 21 - 10);
    for (int k = tid; k < BP_W * BP_H; k += 256) {
        const int ty = k / BP_W, tx = k % BP_W;
        const int sx = clampi(x0 - 10 + tx, 0, img.w - 1), sy = clampi(y0 - 10 + ty, 0, img.h - 1);
        const S* q = pca.px(sx, sy);
        if constexpr (is_half<S>::value) {
            const uint4 u = *reinterpret_cast<const uint4*>(q);
            const float2 a0 = __half22float2(u2h_(u.x)), a1 = __half22float2(u2h_(u.y));
            const float2 a2 = __half22float2(u2h_(u.z)), a3 = __half22float2(u2h_(u.w));
            sm.pca[k][0] = make_float4(a0.x, a0.y, a1.x, a1.y);
            sm.pca[k][1] = make_float4(a2.x, a2.y, a3.x, a3.y);
        } else {
            const float4* q4 = reinterpret_cast<const float4*>(q);
            sm.pca[k][0] = q4[0];
            sm.pca[k][1] = q4[1];
        }
        const f4 p = ld4<S>(img.px(sx, sy));
        sm.ycc[k] = make_float4(p.x, p.y, p.z, 0.f);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, yu = y0 + 2 * threadIdx.y;
    const float kLog2e = 1.4426950408889634f, sq = sqrtf(2.f * kLog2e);
    BmPlainPix pix[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const int c = (2 * threadIdx.y + p + 10) * BP_W + threadIdx.x + 10;
        const float4 in = sm.ycc[c];
        const BmConst k = bm_const<S>(a, grad, img.w, img.h, min(x, img.w - 1), min(yu + p, img.h - 1), in.x, in.y, in.z);
        BmPlainPix& P = pix[p];
        P.p0 = sm.pca[c][0];
        P.p1 = sm.pca[c][1];
        P.kl = -2.f * kLog2e * k.s * k.s;
        P.c1 = sq * k.c1;
        P.c2 = sq * k.c2;
        P.o1 = P.c1 * in.y;
        P.o2 = P.c2 * in.z;
    }
    float acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int col = threadIdx.x, row0 = 2 * threadIdx.y;
    bmp_row<true, false>(sm, row0 * BP_W + col, 0, pix[0], pix[1], acc);
    for (int r = 1; r <= 20; r++) bmp_row<true, true>(sm, (row0 + r) * BP_W + col, r, pix[0], pix[1], acc);
    bmp_row<false, true>(sm, (row0 + 21) * BP_W + col, 21, pix[0], pix[1], acc);
    if (x < out.w) {
        if (yu < out.h) st4<S>(out.px(x, yu), f4{acc[0] / acc[3], acc[1] / acc[4], acc[2] / acc[4], acc[3]});
        if (yu + 1 < out.h) st4<S>(out.px(x, yu + 1), f4{acc[5] / acc[8], acc[6] / acc[9], acc[7] / acc[9], acc[8]});
        if (a.nc_out) {
            if (yu < out.h) a.nc_out[size_t(yu) * out.w + x] = acc[4];
            if (yu + 1 < out.h) a.nc_out[size_t(yu + 1) * out.w + x] = acc[9];
        }
    }
}

// ============================================================ FP16-storage path
// Four vertically adjacent pixels per thread (they share 18 of 24 window
// rows; a staged neighbour feeds 3.5 taps on average), tile 32 x 32, 256
// threads. Shared memory per window position: the PCA coefficients minus
// the tile-centre pixel's, as 8 halves, and (Y, Cb, Cr, |q'|^2) in FP32.
//   * |p - q|^2 = |p'|^2 + |q'|^2 - 2 p'.q' (an 8-FMA dot product, the
//     -2 kl luma scale folded into the centre's coefficients); the
//     centring keeps the cancellation error at FP32 rounding of the local
//     variation of the coefficients;
//   * lw is carried scaled by sqrt(2 log2 e), so the chroma exponent is
//     three FMAs with log2(sw) folded in as the addend, and the luma weight
//     is sw / sqrt(2 log2 e) times it;
//   * both exponentials are ex2.approx (the reference uses half-precision
//     exp under fast math here).
constexpr int BX_TX = 32, BX_W = BX_TX + 20;
// tile variants: TY thread rows of NP vertically adjacent pixels (NP = 4:
// two pixel pairs per thread, NP = 2: one), tiles of 32 x (NP TY) = 32 x 32
// or 32 x 16 pixels; the autotuner picks one per level size
// (launch_block_match). Variant code 10 TY + NP: 84, 44, 82, 162.
template <int TY, int NP>
struct BxTile {
    static constexpr int H = NP * TY + 20;  // window rows staged
    static constexpr int LH = H + 4;        // luma rows staged
    static constexpr int THREADS = BX_TX * TY;
    static constexpr int MIN_BLOCKS = THREADS >= 512 ? 1 : (NP == 4 && TY == 8 ? 2 : 3);
    static_assert(NP == 2 || NP == 4, "one or two pixel pairs per thread");
    static_assert(NP * TY == 16 || NP * TY == 32, "tile heights divide the 32-row centring tiles");
};

// ---------------------------------------------------------------- FFMA2 form
// The four pixels of a thread are taken as two pairs, (p0, p1) and
// (p2, p3), and every per-pixel FP32 operation of a pair is issued as one
// packed FP32x2 instruction (fma/mul/add .rn.f32x2, sm_100a). The neighbour's values enter as broadcast pairs. A pair's
// spatial weights come from one float4 of a 22 x 21 table indexed by the
// pair's first window row (rows outside a pixel's window carry weight 0 and
// log-weight -inf, which zero both of its weights).
typedef unsigned long long u64;

__device__ __forceinline__ u64 pk2(float a, float b) {
    u64 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk2(u64 r, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
    u64 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
    u64 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ u64 add2(u64 a, u64 b) {
    u64 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

template <int H>
struct BmPairSmem {
    uint4 pca[H * BX_W];   // q - c, 8 halves
    float4 ycc[H * BX_W];  // Y, Cb, Cr, |q - c|^2
    float4 sp[22 * 21];       // (sw(j)/sqrt(lk), sw(j-1)/sqrt(lk), -log2 sw(j), -log2 sw(j-1)), j = table row
};

struct BmPair {  // two pixels, each member of a pair register = one pixel
    u64 p[8];             // -2 kl (p - c), per component
    u64 kl, base;         // luma exponent terms
    u64 c1, c2, no1, no2; // chroma: e = c * v - o  (no = -o)
};

template <bool A, bool B, class Sm>
__device__ __forceinline__ void bmp2_row(const Sm& sm, int base, int r, const BmPair& pa, const BmPair& pb,
                                         u64 (&acc)[2][5]) {
    // unrolled 3 of the row's 21 taps: 0.9% faster per 12 MP frame than 7,
    // 1.2% than 1, 1.6% than all 21 (which spills)
#pragma unroll 3
    for (int i = 0; i < 21; i++) {
        const uint4 u = sm.pca[base + i];
        const float2 a0 = __half22float2(u2h_(u.x)), a1 = __half22float2(u2h_(u.y));
        const float2 a2 = __half22float2(u2h_(u.z)), a3 = __half22float2(u2h_(u.w));
        const float4 y = sm.ycc[base + i];
        const u64 q[8] = {pk2(a0.x, a0.x), pk2(a0.y, a0.y), pk2(a1.x, a1.x), pk2(a1.y, a1.y),
                          pk2(a2.x, a2.x), pk2(a2.y, a2.y), pk2(a3.x, a3.x), pk2(a3.y, a3.y)};
        const u64 yy = pk2(y.x, y.x), cb = pk2(y.y, y.y), cr = pk2(y.z, y.z), nn = pk2(y.w, y.w);
        auto pair = [&](const BmPair& P, const float4 s, u64 (&ac)[5]) {
            // ex = kl |q'|^2 - 2 kl p'.q' + base: the -2 kl scale rides in the
            // stored coefficients and base starts the dot-product chain
            u64 dot = fma2(q[0], P.p[0], P.base);
#pragma unroll
            for (int c = 1; c < 8; c++) dot = fma2(q[c], P.p[c], dot);
            const u64 ex = fma2(P.kl, nn, dot);
            float e0, e1;
            upk2(ex, e0, e1);
            float l0, l1;
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(l0) : "f"(fminf(e0, 2.f)));
            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(l1) : "f"(fminf(e1, 2.f)));
            const u64 lws = pk2(l0, l1);
            const u64 d1 = fma2(P.c1, cb, P.no1), d2 = fma2(P.c2, cr, P.no2);
            // q = lws^2 + d1^2 + d2^2 - log2 sw;  wc = exp2(-q)
            const u64 q = fma2(lws, lws, fma2(d1, d1, fma2(d2, d2, pk2(s.z, s.w))));
            float n0, n1;
            upk2(q, n0, n1);
            const float w0 = ex2_approx(-n0), w1 = ex2_approx(-n1);
            const u64 wc = pk2(w0, w1);
            const u64 wy = mul2(pk2(s.x, s.y), lws);
            ac[0] = fma2(wy, yy, ac[0]);
            ac[1] = fma2(wc, cb, ac[1]);
            ac[2] = fma2(wc, cr, ac[2]);
            ac[3] = add2(ac[3], wy);
            ac[4] = add2(ac[4], wc);
        };
        if (A) pair(pa, sm.sp[r * 21 + i], acc[0]);
        if (B) pair(pb, sm.sp[(r - 2) * 21 + i], acc[1]);
    }
}

// pcaProjection (demosaic.metal:774-796) fused into the tile producer: the
// 5x5 luma patch of every window position times the 25 x 8 basis, as FP16
// tensor-core MMAs (mma.sync m16n8k16, FP32 accumulate). 52 x 52 = 2704
// positions = 169 chunks of 16 rows; K = 25 padded to 32 (two k-steps);
// N = the 8 components. The luma tile (window region + 2) is staged once.
constexpr int BX_LW = BX_W + 4;  // luma tile width, origin (x0 - 12, y0 - 12)

__device__ __forceinline__ uint32_t h2u(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// shared memory of one pair-form tile: the staged window region, the
// centring vector and basis, then the luma tile (BX_LH x BX_LW halves)
template <int TY, int NP>
struct BmPairTileSmem {
    BmPairSmem<BxTile<TY, NP>::H> w;
    float cen[8];
    float bsm[25][8];
};
template <int TY, int NP>
constexpr size_t bm_pair_smem_bytes() {
    return sizeof(BmPairTileSmem<TY, NP>) + sizeof(__half) * BX_LW * BxTile<TY, NP>::LH;
}

// One tile (origin x0, y0) of the pair form by TY x 32 threads; the thread
// is (tcol, trow) of the tile. Shared by the stream kernel and the
// persistent kernel's block-matching tasks.
template <int TY, int NP>
__device__ __forceinline__ void bm_pair_tile(int x0, int y0, int tcol, int trow, const Plane<__half, 4>& img,
                                             const Plane<__half, 2>& grad, const float* __restrict__ basis,
                                             const Plane<__half, 4>& out, const BlockMatchArgs& a,
                                             unsigned char* smem_raw) {
    using T = BxTile<TY, NP>;
    constexpr int BX_H = T::H, BX_LH = T::LH, NT = T::THREADS, BX_NP = NP;
    BmPairTileSmem<TY, NP>& st = *reinterpret_cast<BmPairTileSmem<TY, NP>*>(smem_raw);
    BmPairSmem<BX_H>& sm = st.w;
    __half* luma = reinterpret_cast<__half*>(smem_raw + sizeof(BmPairTileSmem<TY, NP>));  // BX_LH x BX_LW
    float* cen = st.cen;
    float (*bsm)[8] = st.bsm;
    const int tid = trow * BX_TX + tcol;
    const float kLog2e = 1.4426950408889634f, lk = 2.f * kLog2e, isq = rsqrtf(lk);
    for (int k = tid; k < 22 * 21; k += NT) {
        const int j = k / 21, i = k % 21 - 10;
        // window row j of the pair's first pixel, j - 1 of its second
        const float w0 = j <= 20 ? spatial_weight(i, j - 10) : 0.f;
        const float w1 = j >= 1 ? spatial_weight(i, j - 11) : 0.f;
        sm.sp[k] = make_float4(w0 * isq, w1 * isq, -log2f(w0), -log2f(w1));
    }
    for (int k = tid; k < 200; k += NT) bsm[k / 8][k % 8] = basis[k];
    for (int k = tid; k < BX_LW * BX_LH; k += NT) {
        const int ty = k / BX_LW, tx = k % BX_LW;
        luma[k] = *img.pxc(x0 - 12 + tx, y0 - 12 + ty);
    }
    for (int k = tid; k < BX_W * BX_H; k += NT) {
        const int ty = k / BX_W, tx = k % BX_W;
        const f4 p = ld4<__half>(img.pxc(x0 - 10 + tx, y0 - 10 + ty));
        sm.ycc[k] = make_float4(p.x, p.y, p.z, 0.f);
    }
    __syncthreads();
    if (tid < 8) {  // centring vector: the coefficients (FP32) of the centre pixel of the
                    // enclosing 32 x 32 tile, so that both tile heights centre and round alike
        const int cx = BX_TX / 2 + 12, cy = 16 + 12 - (y0 % 32);  // luma-tile coordinates
        float c = 0.f;
        for (int k = 0; k < 25; k++) c += bsm[k][tid] * __half2float(luma[(cy + k / 5 - 2) * BX_LW + cx + k % 5 - 2]);
        cen[tid] = c;
    }
    // B fragments (basis, k x n, "col" layout): rows 2t, 2t+1, 2t+8, 2t+9 of column g, per k-step
    const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
    uint32_t bf[2][2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        auto bk = [&](int k) { return k < 25 ? bsm[k][g] : 0.f; };
        const int k0 = 16 * s + 2 * t;
        bf[s][0] = h2u(__floats2half2_rn(bk(k0), bk(k0 + 1)));
        bf[s][1] = h2u(__floats2half2_rn(bk(k0 + 8), bk(k0 + 9)));
    }
    __syncthreads();
    uint32_t* pca32 = reinterpret_cast<uint32_t*>(sm.pca);  // [position][4] half2
    for (int ch = warp; ch < (BX_W * BX_H) / 16; ch += TY) {
        const int m0 = ch * 16 + g, m1 = m0 + 8;  // the two rows of this thread
        // patch centre in the luma tile: the clamped image position of the
        // window position, as a clamped read of a projected plane would see
        auto lidx = [&](int m) {
            const int px = clampi(x0 - 10 + m % BX_W, 0, img.w - 1) - (x0 - 12);
            const int py = clampi(y0 - 10 + m / BX_W, 0, img.h - 1) - (y0 - 12);
            return py * BX_LW + px;
        };
        const int l0 = lidx(m0), l1 = lidx(m1);
        auto av = [&](int l, int k) {  // patch element k of the position at luma index l
            return k < 25 ? luma[l + (k / 5 - 2) * BX_LW + (k % 5 - 2)] : __float2half(0.f);
        };
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int k0 = 16 * s + 2 * t;
            const uint32_t a0 = h2u(__halves2half2(av(l0, k0), av(l0, k0 + 1)));
            const uint32_t a1 = h2u(__halves2half2(av(l1, k0), av(l1, k0 + 1)));
            const uint32_t a2 = h2u(__halves2half2(av(l0, k0 + 8), av(l0, k0 + 9)));
            const uint32_t a3 = h2u(__halves2half2(av(l1, k0 + 8), av(l1, k0 + 9)));
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                "{%0,%1,%2,%3};"
                : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(bf[s][0]), "r"(bf[s][1]));
        }
        // rows m0 (c0, c1) and m1 (c2, c3), components 2t, 2t+1; centre, round, store
        const __half2 h0 = __floats2half2_rn(c[0] - cen[2 * t], c[1] - cen[2 * t + 1]);
        const __half2 h1 = __floats2half2_rn(c[2] - cen[2 * t], c[3] - cen[2 * t + 1]);
        pca32[m0 * 4 + t] = h2u(h0);
        pca32[m1 * 4 + t] = h2u(h1);
        const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
        float n0 = f0.x * f0.x + f0.y * f0.y, n1 = f1.x * f1.x + f1.y * f1.y;
        n0 += __shfl_xor_sync(0xffffffffu, n0, 1);
        n0 += __shfl_xor_sync(0xffffffffu, n0, 2);
        n1 += __shfl_xor_sync(0xffffffffu, n1, 1);
        n1 += __shfl_xor_sync(0xffffffffu, n1, 2);
        if (t == 0) {
            sm.ycc[m0].w = n0;
            sm.ycc[m1].w = n1;
        }
    }
    __syncthreads();
    const int x = x0 + tcol, y = y0 + BX_NP * trow;
    float pc[BX_NP][8], kl[BX_NP], base[BX_NP], c1[BX_NP], c2[BX_NP], o1[BX_NP], o2[BX_NP];
#pragma unroll
    for (int p = 0; p < BX_NP; p++) {
        const int c = (BX_NP * trow + p + 10) * BX_W + tcol + 10;
        const float4 in = sm.ycc[c];
        const uint4 u = sm.pca[c];
        const float2 a0 = __half22float2(u2h_(u.x)), a1 = __half22float2(u2h_(u.y));
        const float2 a2 = __half22float2(u2h_(u.z)), a3 = __half22float2(u2h_(u.w));
        pc[p][0] = a0.x; pc[p][1] = a0.y; pc[p][2] = a1.x; pc[p][3] = a1.y;
        pc[p][4] = a2.x; pc[p][5] = a2.y; pc[p][6] = a3.x; pc[p][7] = a3.y;
        const BmConst k =
            bm_const<__half>(a, grad, img.w, img.h, min(x, img.w - 1), min(y + p, img.h - 1), in.x, in.y, in.z);
        kl[p] = fmaxf(-2.f * kLog2e * k.s * k.s, -1e30f);
        base[p] = fmaf(kl[p], in.w, 0.5f * log2f(lk));
        const float sq = sqrtf(lk);
        c1[p] = sq * k.c1;
        c2[p] = sq * k.c2;
        o1[p] = c1[p] * in.y;
        o2[p] = c2[p] * in.z;
    }
    BmPair PP[NP / 2];
#pragma unroll
    for (int q = 0; q < NP / 2; q++) {
        for (int c = 0; c < 8; c++) PP[q].p[c] = pk2(-2.f * kl[2 * q] * pc[2 * q][c], -2.f * kl[2 * q + 1] * pc[2 * q + 1][c]);
        PP[q].kl = pk2(kl[2 * q], kl[2 * q + 1]);
        PP[q].base = pk2(base[2 * q], base[2 * q + 1]);
        PP[q].c1 = pk2(c1[2 * q], c1[2 * q + 1]);
        PP[q].c2 = pk2(c2[2 * q], c2[2 * q + 1]);
        PP[q].no1 = pk2(-o1[2 * q], -o1[2 * q + 1]);
        PP[q].no2 = pk2(-o2[2 * q], -o2[2 * q + 1]);
    }
    u64 acc[2][5];
    for (int k = 0; k < 5; k++) acc[0][k] = acc[1][k] = pk2(0.f, 0.f);
    const int col = tcol, row0 = BX_NP * trow;
    auto rb = [&](int r) { return (row0 + r) * BX_W + col; };
    const BmPair& PA = PP[0];
    const BmPair& PB = PP[NP / 2 - 1];  // the second pair (unused when NP = 2)
    if constexpr (NP == 4) {
        bmp2_row<true, false>(sm, rb(0), 0, PA, PB, acc);
        bmp2_row<true, false>(sm, rb(1), 1, PA, PB, acc);
        for (int r = 2; r <= 21; r++) bmp2_row<true, true>(sm, rb(r), r, PA, PB, acc);
        bmp2_row<false, true>(sm, rb(22), 22, PA, PB, acc);
        bmp2_row<false, true>(sm, rb(23), 23, PA, PB, acc);
    } else {
        for (int r = 0; r <= 21; r++) bmp2_row<true, false>(sm, rb(r), r, PA, PB, acc);
    }
    float v[2][5][2];
    for (int q = 0; q < 2; q++)
        for (int k = 0; k < 5; k++) upk2(acc[q][k], v[q][k][0], v[q][k][1]);
    if (x < out.w) {
#pragma unroll
        for (int p = 0; p < BX_NP; p++) {
            const int q = p >> 1, m = p & 1;
            if (y + p < out.h)
                st4<__half>(out.px(x, y + p), f4{v[q][0][m] / v[q][3][m], v[q][1][m] / v[q][4][m],
                                                 v[q][2][m] / v[q][4][m], v[q][3][m]});
        }
    }
}


template <int TY, int NP>
__global__ void __launch_bounds__(BxTile<TY, NP>::THREADS, BxTile<TY, NP>::MIN_BLOCKS)
    k_block_match_pair(Plane<__half, 4> img, Plane<__half, 2> grad, const float* __restrict__ basis,
                       Plane<__half, 4> out, BlockMatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bm_pair_tile<TY, NP>(blockIdx.x * BX_TX, blockIdx.y * (NP * TY), threadIdx.x, threadIdx.y, img, grad, basis, out,
                         a, smem_raw);
}

template <int TY, int NP>
static void launch_pair(Plane<__half, 4> img, Plane<__half, 2> grad, const float* basis, Plane<__half, 4> out,
                        const BlockMatchArgs& a, cudaStream_t s) {
    const size_t smem = bm_pair_smem_bytes<TY, NP>();
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_block_match_pair<TY, NP>), int(smem));
    dim3 b(BX_TX, TY);
    dim3 g((img.w + BX_TX - 1) / BX_TX, (img.h + NP * TY - 1) / (NP * TY));
    k_block_match_pair<TY, NP><<<g, b, smem, s>>>(img, grad, basis, out, a);
}

// the pair kernel's variants by code (10 TY + NP)
static constexpr int kBmVariants[4] = {84, 44, 82, 162};

static void launch_pair_variant(int code, Plane<__half, 4> img, Plane<__half, 2> grad, const float* basis,
                                Plane<__half, 4> out, const BlockMatchArgs& a, cudaStream_t s) {
    switch (code) {
        case 44: launch_pair<4, 4>(img, grad, basis, out, a, s); break;
        case 82: launch_pair<8, 2>(img, grad, basis, out, a, s); break;
        case 162: launch_pair<16, 2>(img, grad, basis, out, a, s); break;
        default: launch_pair<8, 4>(img, grad, basis, out, a, s); break;
    }
}

// ============================================================ FP16-storage path, tensor-core form
// The window sums as matrix products on the tensor cores, one warp per
// group of 16 pixels (a 4 x 4 block, the block shape whose windows overlap
// most: their union is 24 x 24 positions, of which each pixel's 21 x 21
// window is 76.6%). The union is walked as 72 tiles of 8 neighbours (24
// rows x 3 row segments). Per tile:
//   * S = -2 p'.q' + |q'|^2 for the 16 pixels x 8 neighbours by one
//     mma.sync m16n8k8 (FP16 in, FP32 accumulate): A holds each pixel's
//     centred coefficients times -2, B the neighbours' centred
//     coefficients, C the neighbours' |q'|^2. The coefficients are stored
//     in FP16 and the scaling by -2 is exact, so the products are exact
//     and the sum is an FP32 sum, as in a scalar FP32 evaluation;
//   * the weights from the accumulator fragment, two neighbours of a pixel
//     at a time: luma exponent kl S + (kl |p'|^2 + log2 sqrt(lk)) by one
//     packed FP32 FMA, both exponentials as ex2.approx.f16x2 (the
//     reference evaluates its weights in half precision,
//     demosaic.metal:851-874), chroma exponent in packed FP32;
//   * the weights, already in the accumulator layout of S, are the A
//     operand of two more MMAs (two tiles per k-step) against B = the
//     neighbours' (Y, 0, 0, 1) and (0, Cb, Cr, 0, 1) columns, which add
//     sum w Y, sum w Cb, sum w Cr and both kernel norms in FP32.
// A neighbour outside a pixel's window has spatial weight 0 (and
// -log2 weight +inf), which zeroes both of its weights. The spatial
// Gaussian is separable: its x part per lane and row segment is held in
// registers, its y part per union row comes from a 27-entry table.
constexpr int BM_T = 32, BM_W = BM_T + 20, BM_N = BM_W * BM_W, BM_LW = BM_W + 4, BM_THREADS = 256;

struct BmMmaSmem {
    uint4 q[BM_N];               // q - c, 8 halves
    float nn[BM_N];              // |q - c|^2
    __half y[BM_N], cb[BM_N], cr[BM_N];
    float lswy[32];              // -log2 of the spatial weight's y part, dy = -13..13 (+inf outside +-10)
    __half swy[32];              // its y part / sqrt(lk) (0 outside)
    __half luma[BM_LW * BM_LW];  // the luma tile of the projection patches, origin (x0 - 12, y0 - 12)
    float cen[8];                // the centring vector
    float bsm[25][8];            // the level's basis
};

__device__ __forceinline__ uint32_t cvt_h2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ uint32_t ex2_h2(uint32_t x) {
    uint32_t r;
    asm("ex2.approx.f16x2 %0, %1;" : "=r"(r) : "r"(x));
    return r;
}
__device__ __forceinline__ uint32_t hmul2_u(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("mul.rn.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ u64 h2_to_f2(uint32_t h) {
    const float2 f = __half22float2(u2h_(h));
    return pk2(f.x, f.y);
}
__device__ __forceinline__ void mma1688(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0, float c0, float c1,
                                        float c2, float c3) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%7,%8,%9,%10};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a0), "r"(a1), "r"(b0), "f"(c0), "f"(c1), "f"(c2), "f"(c3));
}
__device__ __forceinline__ uint32_t hmin2_u(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ void mma16816_acc(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                             uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Per pixel row of a lane (pixel g or g + 8 of the group): the constants
// of its two neighbours' weights, as packed pairs.
struct BmRow {
    u64 kl, base;          // luma exponent kl S + base
    u64 c1, c2, no1, no2;  // chroma: d = c v - o
};

// The weights of one pixel row for the lane's two neighbours of a tile:
// (wy, wc) as half2 pairs, from its S pair (s0, s1).
__device__ __forceinline__ void bm_weights(const BmRow& R, float s0, float s1, u64 cbf, u64 crf, u64 lsw,
                                           uint32_t swp, uint32_t& wy, uint32_t& wc) {
    float e0, e1;
    upk2(fma2(R.kl, pk2(s0, s1), R.base), e0, e1);
    // sqrt(lk) lw for both neighbours; the exponent is at most log2 sqrt(lk)
    // but for rounding, and is held below 2 as the FP32 kernel holds it
    const uint32_t lws = ex2_h2(hmin2_u(cvt_h2(e0, e1), 0x40004000u));
    const u64 lf = h2_to_f2(lws);
    const u64 d1 = fma2(R.c1, cbf, R.no1), d2 = fma2(R.c2, crf, R.no2);
    float q0, q1;
    upk2(fma2(lf, lf, fma2(d1, d1, fma2(d2, d2, lsw))), q0, q1);
    wc = ex2_h2(cvt_h2(-q0, -q1));                    // sw cw
    wy = hmul2_u(lws, swp);                           // sw lw
}

// One 32 x 32 tile (origin x0, y0) by a block of BM_THREADS threads.
__device__ __forceinline__ void bm_mma_tile(int x0, int y0, const Plane<__half, 4>& img, const Plane<__half, 2>& grad,
                                            const float* __restrict__ basis, const Plane<__half, 4>& out,
                                            const BlockMatchArgs& a, BmMmaSmem& sm) {
    float* cen = sm.cen;
    float (*bsm)[8] = sm.bsm;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
    const float kLog2e = 1.4426950408889634f, lk = 2.f * kLog2e, isq = rsqrtf(lk);
    // ---- staging: spatial y table, basis, luma tile, Y/Cb/Cr of the window region
    if (tid < 32) {
        const int dy = tid - 13;
        const bool in = dy >= -10 && dy <= 10;
        const float w = in ? spatial_weight(0, dy) : 0.f;
        sm.lswy[tid] = in ? -log2f(w) : __int_as_float(0x7f800000);
        sm.swy[tid] = __float2half_rn(w * isq);
    }
    for (int k = tid; k < 200; k += BM_THREADS) bsm[k / 8][k % 8] = basis[k];
    for (int k = tid; k < BM_LW * BM_LW; k += BM_THREADS) {
        const int ty = k / BM_LW, tx = k % BM_LW;
        sm.luma[k] = *img.pxc(x0 - 12 + tx, y0 - 12 + ty);
    }
    for (int k = tid; k < BM_N; k += BM_THREADS) {
        const int ty = k / BM_W, tx = k % BM_W;
        const __half* p = img.pxc(x0 - 10 + tx, y0 - 10 + ty);
        sm.y[k] = p[0];
        sm.cb[k] = p[1];
        sm.cr[k] = p[2];
    }
    __syncthreads();
    if (tid < 8) {  // centring vector: the coefficients (FP32) of the tile's centre pixel
        const int cx = BM_T / 2 + 12, cy = BM_T / 2 + 12;
        float c = 0.f;
        for (int k = 0; k < 25; k++) c += bsm[k][tid] * __half2float(sm.luma[(cy + k / 5 - 2) * BM_LW + cx + k % 5 - 2]);
        cen[tid] = c;
    }
    // pcaProjection (demosaic.metal:774-796) of every staged position:
    // 16 positions x 5x5 patch (K = 25 padded to 32) x 25x8 basis per MMA
    uint32_t bf[2][2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        auto bk = [&](int k) { return k < 25 ? bsm[k][g] : 0.f; };
        const int k0 = 16 * s + 2 * t;
        bf[s][0] = h2u(__floats2half2_rn(bk(k0), bk(k0 + 1)));
        bf[s][1] = h2u(__floats2half2_rn(bk(k0 + 8), bk(k0 + 9)));
    }
    __syncthreads();
    uint32_t* q32 = reinterpret_cast<uint32_t*>(sm.q);  // [position][4] half2
    for (int ch = warp; ch < BM_N / 16; ch += BM_THREADS / 32) {
        const int m0 = ch * 16 + g, m1 = m0 + 8;
        auto lidx = [&](int m) {  // the clamped image position of window position m, in the luma tile
            const int px = clampi(x0 - 10 + m % BM_W, 0, img.w - 1) - (x0 - 12);
            const int py = clampi(y0 - 10 + m / BM_W, 0, img.h - 1) - (y0 - 12);
            return py * BM_LW + px;
        };
        const int l0 = lidx(m0), l1 = lidx(m1);
        auto av = [&](int l, int k) { return k < 25 ? sm.luma[l + (k / 5 - 2) * BM_LW + (k % 5 - 2)] : __float2half(0.f); };
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int k0 = 16 * s + 2 * t;
            mma16816_acc(c, h2u(__halves2half2(av(l0, k0), av(l0, k0 + 1))), h2u(__halves2half2(av(l1, k0), av(l1, k0 + 1))),
                         h2u(__halves2half2(av(l0, k0 + 8), av(l0, k0 + 9))),
                         h2u(__halves2half2(av(l1, k0 + 8), av(l1, k0 + 9))), bf[s][0], bf[s][1]);
        }
        const __half2 h0 = __floats2half2_rn(c[0] - cen[2 * t], c[1] - cen[2 * t + 1]);
        const __half2 h1 = __floats2half2_rn(c[2] - cen[2 * t], c[3] - cen[2 * t + 1]);
        q32[m0 * 4 + t] = h2u(h0);
        q32[m1 * 4 + t] = h2u(h1);
        const float2 f0 = __half22float2(h0), f1 = __half22float2(h1);
        float n0 = f0.x * f0.x + f0.y * f0.y, n1 = f1.x * f1.x + f1.y * f1.y;
        n0 += __shfl_xor_sync(0xffffffffu, n0, 1);
        n0 += __shfl_xor_sync(0xffffffffu, n0, 2);
        n1 += __shfl_xor_sync(0xffffffffu, n1, 1);
        n1 += __shfl_xor_sync(0xffffffffu, n1, 2);
        if (t == 0) {
            sm.nn[m0] = n0;
            sm.nn[m1] = n1;
        }
    }
    __syncthreads();

    // ---- lane constants: the x part of the spatial weight for the lane's
    //      neighbour pair (2t, 2t + 1) of each row segment, pixel column g % 4
    const int pxl = g & 3;
    u64 lswx[3];
    uint32_t swx[3];
#pragma unroll
    for (int s = 0; s < 3; s++) {
        float l[2], w[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int dx = 8 * s + 2 * t + e - pxl - 10;
            const bool in = dx >= -10 && dx <= 10;
            w[e] = in ? spatial_weight(dx, 0) : 0.f;
            l[e] = in ? -log2f(w[e]) : __int_as_float(0x7f800000);
        }
        lswx[s] = pk2(l[0], l[1]);
        swx[s] = cvt_h2(w[0], w[1]);
    }
    const uint32_t ONE2 = 0x3c003c00u;  // half2 (1, 1)
    const __half* ysrc = sm.y;  // the luma B column (lanes g == 0)

    // ---- 4 x 4 pixel groups: 64 per tile, warp w takes groups w, w + 8, ...
    for (int grp = warp; grp < (BM_T / 4) * (BM_T / 4); grp += BM_THREADS / 32) {
        const int gx = (grp % (BM_T / 4)) * 4, gy = (grp / (BM_T / 4)) * 4;  // tile coordinates
        // the lane's two pixels: rows g and g + 8 of the group = (g % 4, g / 4) and (g % 4, g / 4 + 2)
        BmRow R[2];
        uint32_t ap[2];  // A fragments: -2 p', components 2t, 2t + 1
        int py[2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
            py[r] = (g >> 2) + 2 * r;
            const int sx = gx + pxl + 10, sy = gy + py[r] + 10;  // staged position of the pixel
            const int pos = sy * BM_W + sx;
            const float in_y = __half2float(sm.y[pos]), in_cb = __half2float(sm.cb[pos]), in_cr = __half2float(sm.cr[pos]);
            const int ix = min(x0 + gx + pxl, img.w - 1), iy = min(y0 + gy + py[r], img.h - 1);
            const BmConst k = bm_const<__half>(a, grad, img.w, img.h, ix, iy, in_y, in_cb, in_cr);
            const float kl = fmaxf(-2.f * kLog2e * k.s * k.s, -1e30f);
            const float base = fmaf(kl, sm.nn[pos], 0.5f * log2f(lk));
            const float sq = sqrtf(lk);
            const float c1 = sq * k.c1, c2 = sq * k.c2;
            R[r].kl = pk2(kl, kl);
            R[r].base = pk2(base, base);
            R[r].c1 = pk2(c1, c1);
            R[r].c2 = pk2(c2, c2);
            R[r].no1 = pk2(-c1 * in_cb, -c1 * in_cb);
            R[r].no2 = pk2(-c2 * in_cr, -c2 * in_cr);
            ap[r] = hmul2_u(q32[pos * 4 + t], 0xc000c000u);  // p' components 2t, 2t + 1, times -2 (exact)
        }
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        // union rows ny = 0..23 (staged rows gy + ny), segments s = 0..2
        // (staged columns gx + 8 s .. + 7): tiles in row-major order, two per k-step
        uint32_t pwy[2], pwc[2], pby, pbc;  // the pending (first) tile of a k-step
#pragma unroll 1
        for (int ny = 0; ny < 24; ny += 2) {
#pragma unroll
            for (int j = 0; j < 6; j++) {
                const int row = ny + j / 3, s = j % 3;
                const int base_pos = (gy + row) * BM_W + gx + 8 * s;
                // B of S: neighbour g's coefficients 2t, 2t + 1
                const uint32_t bq = q32[(base_pos + g) * 4 + t];
                const float2 nnp = *reinterpret_cast<const float2*>(&sm.nn[base_pos + 2 * t]);
                float S[4];
                mma1688(S, ap[0], ap[1], bq, nnp.x, nnp.y, nnp.x, nnp.y);
                const uint32_t cbh = *reinterpret_cast<const uint32_t*>(&sm.cb[base_pos + 2 * t]);
                const uint32_t crh = *reinterpret_cast<const uint32_t*>(&sm.cr[base_pos + 2 * t]);
                const uint32_t yh = *reinterpret_cast<const uint32_t*>(&ysrc[base_pos + 2 * t]);
                const u64 cbf = h2_to_f2(cbh), crf = h2_to_f2(crh);
                uint32_t wy[2], wc[2];
#pragma unroll
                for (int r = 0; r < 2; r++) {
                    const int dyi = row - py[r] - 10 + 13;  // 0..26
                    const float ly = sm.lswy[dyi];
                    const __half sy = sm.swy[dyi];
                    const u64 lsw = add2(lswx[s], pk2(ly, ly));
                    const uint32_t swp = hmul2_u(swx[s], h2u(__halves2half2(sy, sy)));
                    bm_weights(R[r], S[2 * r], S[2 * r + 1], cbf, crf, lsw, swp, wy[r], wc[r]);
                }
                // B columns of the sums: luma (Y, 0, 0, 1, 0..), chroma (0, Cb, Cr, 0, 1, 0..)
                const uint32_t by = g == 0 ? yh : (g == 3 ? ONE2 : 0u);
                const uint32_t bc = g == 1 ? cbh : (g == 2 ? crh : (g == 4 ? ONE2 : 0u));
                if ((j & 1) == 0) {
                    pwy[0] = wy[0]; pwy[1] = wy[1]; pwc[0] = wc[0]; pwc[1] = wc[1]; pby = by; pbc = bc;
                } else {
                    mma16816_acc(acc, pwy[0], pwy[1], wy[0], wy[1], pby, by);
                    mma16816_acc(acc, pwc[0], pwc[1], wc[0], wc[1], pbc, bc);
                }
            }
        }
        // acc: rows g, g + 8; columns 2t, 2t + 1. Column 0 sum wy Y, 1 sum wc Cb,
        // 2 sum wc Cr, 3 sum wy, 4 sum wc: gather to lane t = 0
        const float a2 = __shfl_down_sync(0xffffffffu, acc[0], 1), a3 = __shfl_down_sync(0xffffffffu, acc[1], 1);
        const float a4 = __shfl_down_sync(0xffffffffu, acc[0], 2);
        const float b2 = __shfl_down_sync(0xffffffffu, acc[2], 1), b3 = __shfl_down_sync(0xffffffffu, acc[3], 1);
        const float b4 = __shfl_down_sync(0xffffffffu, acc[2], 2);
        if (t == 0) {
            const int ox = x0 + gx + pxl;
            if (ox < out.w) {
                const int oy0 = y0 + gy + py[0], oy1 = y0 + gy + py[1];
                if (oy0 < out.h) st4<__half>(out.px(ox, oy0), f4{acc[0] / a3, acc[1] / a4, a2 / a4, a3});
                if (oy1 < out.h) st4<__half>(out.px(ox, oy1), f4{acc[2] / b3, acc[3] / b4, b2 / b4, b3});
            }
        }
    }
}

__global__ void __launch_bounds__(BM_THREADS, 2)
    k_block_match_mma(Plane<__half, 4> img, Plane<__half, 2> grad, const float* __restrict__ basis,
                      Plane<__half, 4> out, BlockMatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bm_mma_tile(blockIdx.x * BM_T, blockIdx.y * BM_T, img, grad, basis, out, a,
                *reinterpret_cast<BmMmaSmem*>(smem_raw));
}

static void launch_mma(Plane<__half, 4> img, Plane<__half, 2> grad, const float* basis, Plane<__half, 4> out,
                       const BlockMatchArgs& a, cudaStream_t s) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_block_match_mma), int(sizeof(BmMmaSmem)));
    dim3 g((img.w + BM_T - 1) / BM_T, (img.h + BM_T - 1) / BM_T);
    k_block_match_mma<<<g, BM_THREADS, sizeof(BmMmaSmem), s>>>(img, grad, basis, out, a);
}

// ============================================================ persistent batch kernel
// PyramidProcessor::denoise (pyramid_processor.cpp:96-172) for every frame
// of a batch in one launch. The host lists the work of every (frame,
// level) as tasks: reconstruct tiles (SN, 64 x 64 pixels), covariance
// partial rows (COV), the eigen-solve (EIG) and block-matching tiles (BM,
// 32 x 32), level by level from the coarsest, all frames' SN / COV / EIG of
// a level before their BM tiles. A block takes the next task from a
// counter, waits until the task's inputs are complete, runs it with the
// same device code as the stream kernels (so the results are
// bit-identical), and counts it done:
//   SN (f, l)  waits for every BM tile of (f, l + 1)  (the coarse denoised image)
//   COV (f, l) waits for every SN tile of (f, l)      (the layer)
//   EIG (f, l) waits for every COV row of (f, l)
//   BM (f, l)  waits for EIG (f, l)                   (the basis; the layer before it)
// Every task a block waits for comes earlier in the list and was taken by a
// running block, so the earliest unfinished task can always run: the order
// cannot deadlock, and the blocks need not be co-resident. A wait is
// bounded: past limit_ns (global timer) the block records the task type
// in *err and every block stops taking tasks; the host reads the word and
// returns GLS_ERR_TIMEOUT.
struct PSmem {
    union {
        alignas(16) unsigned char bm[bm_pair_smem_bytes<8, 4>()];  // a 32 x 32 tile of the pair form
        EigenSmem eig;
        CovSmem cov;
    };
};

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The two calls below take the block's shared memory from the extern
// array itself, not as a pointer argument: across a call boundary a pointer
// is generic, and the tile's staged reads would compile to generic loads
// instead of shared-memory loads. Their level arguments are copied out of
// the descriptor once, as a kernel's parameters would be.

// the rarely taken eigen-solve as a call of its own, so that its registers
// do not weigh on the block-matching path
__device__ __noinline__ void persistent_eigen(const PLevel& L) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pca_eigen_block(L.part, L.n_cov, (L.layer.w / 8) * (L.layer.h / 8), L.basis, L.status,
                    reinterpret_cast<PSmem*>(smem_raw)->eig);
}

// a block-matching task: one 32 x 32 tile of the default (pair-form)
// matcher in its 8 x 4 variant, the same bits as every stream variant
__device__ __noinline__ void persistent_bm(const PLevel& L, uint32_t item) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Plane<__half, 4> layer = L.layer, den = L.den;
    const Plane<__half, 2> grad = L.grad;
    const float* basis = L.basis;
    const BlockMatchArgs ba = L.ba;
    const int tx = int(item) % L.tiles_x, ty = int(item) / L.tiles_x;
    bm_pair_tile<8, 4>(tx * BM_T, ty * BM_T, threadIdx.x & 31, threadIdx.x >> 5, layer, grad, basis, den, ba,
                       reinterpret_cast<PSmem*>(smem_raw)->bm);
}

__global__ void __launch_bounds__(BM_THREADS, 2)
    k_pyramid_persistent(const PTask* __restrict__ tasks, int n_tasks, const PLevel* __restrict__ lv,
                         PCounters* __restrict__ cnt, int* __restrict__ next, int* __restrict__ err, long long limit_ns) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PSmem& sm = *reinterpret_cast<PSmem*>(smem_raw);
    __shared__ int s_task, s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_task = ld_acquire(err) ? n_tasks : atomicAdd(next, 1);
        __syncthreads();
        const int ti = s_task;
        if (ti >= n_tasks) break;
        const PTask tk = tasks[ti];
        const uint32_t type = tk.item >> 30, item = tk.item & kPTaskItemMask;
        const PLevel& L = lv[tk.lev];
        if (threadIdx.x == 0) {
            // the counter this task waits on and its target (none: -1)
            const int* c = nullptr;
            int target = 0;
            if (type == PT_SN) {
                c = &cnt[L.coarser].bm;
                target = lv[L.coarser].n_bm;
            } else if (type == PT_COV) {
                if (L.n_sn > 0) {
                    c = &cnt[tk.lev].sn;
                    target = L.n_sn;
                }
            } else if (type == PT_EIG) {
                c = &cnt[tk.lev].cov;
                target = L.n_cov;
            } else {
                c = &cnt[tk.lev].eig;
                target = 1;
            }
            int ok = 1;
            if (c && ld_acquire(c) < target) {
                const long long t0 = global_ns();
                unsigned ns = 32;
                while (ld_acquire(c) < target) {
                    if (ld_acquire(err) || global_ns() - t0 > limit_ns) {
                        atomicCAS(err, 0, int(1 + type));
                        ok = 0;
                        break;
                    }
                    __nanosleep(ns);
                    ns = ns < 2048 ? 2 * ns : ns;
                }
            }
            __threadfence();
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) break;
        int* done;
        if (type == PT_SN) {
            const int tx = item % L.sn_tiles_x, ty = item / L.sn_tiles_x;
            for (int k = threadIdx.x; k < kPSnTile * kPSnTile; k += BM_THREADS) {
                const int x = tx * kPSnTile + k % kPSnTile, y = ty * kPSnTile + k / kPSnTile;
                if (x < L.img.w && y < L.img.h)
                    subtract_noise_px<__half>(L.img, L.coarse, L.coarse_den, L.grad, L.layer, L.sa, L.rx, L.ry, x, y);
            }
            done = &cnt[tk.lev].sn;
        } else if (type == PT_COV) {
            const int c0 = int(item) * L.cov_group;
            pca_cov_row<__half>(L.layer, L.part + size_t(item) * kPcaAcc, c0, min(c0 + L.cov_group, L.chunks), sm.cov);
            done = &cnt[tk.lev].cov;
        } else if (type == PT_EIG) {
            persistent_eigen(L);
            done = &cnt[tk.lev].eig;
        } else {
            persistent_bm(L, item);
            done = &cnt[tk.lev].bm;
        }
        __syncthreads();  // the task's writes, and its shared memory, are finished
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(done, 1);
        }
    }
}

int persistent_grid(int device) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_pyramid_persistent), int(sizeof(PSmem)));
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pyramid_persistent, BM_THREADS, sizeof(PSmem)) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return 0;
    return per_sm * sms;
}

void launch_pyramid_persistent(const PTask* tasks, int n, const PLevel* lv, PCounters* cnt, int* next, int* err,
                               long long limit_ns, int grid, cudaStream_t s) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_pyramid_persistent), int(sizeof(PSmem)));
    k_pyramid_persistent<<<grid, BM_THREADS, sizeof(PSmem), s>>>(tasks, n, lv, cnt, next, err, limit_ns);
}

// Tile autotuner of the FP16 block matcher. Its variants (thread rows x
// pixels per thread: 8 x 4 and 16 x 2 for 32 x 32 tiles, 4 x 4 and 8 x 2
// for 32 x 16) compute identical results (the same per-pixel arithmetic,
// pairs of pixels in packed FP32, and the same centring), so the choice only
// changes speed: 32 x 32 tiles amortise the staged halo better, 32 x 16
// tiles fill the GPU on small pyramid levels, and one pair per thread
// trades the reuse of a staged neighbour for occupancy. The first call for
// a level size times every variant on the caller's stream (leaving the
// result in `out`) and keeps the fastest; later calls reuse the choice, and
// so do calls made while the stream is being captured into a graph
// (default 8 x 4 for a size not timed yet). GLS_BM_TILE=84, 44, 82 or 162 in
// the environment (or 8 / 4 for 84 / 44) fixes the variant.
static std::mutex g_tile_mu;
static std::map<std::pair<int, int>, int> g_tile_choice;

int bm_tile_list(int* whty, int max) {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    int n = 0;
    for (const auto& kv : g_tile_choice) {
        if (n < max) {
            whty[3 * n] = kv.first.first;
            whty[3 * n + 1] = kv.first.second;
            whty[3 * n + 2] = kv.second;
        }
        n++;
    }
    return n;
}

template <class Run>
static int bm_tile_variant(int w, int h, Run&& run_variant, cudaStream_t s) {
    static const int forced = [] {
        const char* e = std::getenv("GLS_BM_TILE");
        const int v = e ? std::atoi(e) : 0;
        if (v == 8) return 84;  // the thread-row counts of the two NP = 4 variants
        if (v == 4) return 44;
        for (int c : kBmVariants)
            if (v == c) return v;
        return 0;
    }();
    if (forced) return forced;
    {
        std::lock_guard<std::mutex> lk(g_tile_mu);
        auto it = g_tile_choice.find({w, h});
        if (it != g_tile_choice.end()) return it->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return 84;
    constexpr int NV = sizeof(kBmVariants) / sizeof(kBmVariants[0]);
    cudaEvent_t e[NV + 1];
    for (auto& ev : e) cudaEventCreate(&ev);
    cudaEventRecord(e[0], s);
    for (int v = 0; v < NV; v++) {
        run_variant(kBmVariants[v]);
        cudaEventRecord(e[v + 1], s);
    }
    int choice = 84;
    if (cudaEventSynchronize(e[NV]) == cudaSuccess) {
        float best = 0.f;
        for (int v = 0; v < NV; v++) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, e[v], e[v + 1]) != cudaSuccess) continue;
            if (v == 0 || t < best) {
                best = t;
                choice = kBmVariants[v];
            }
        }
    }
    for (auto& ev : e) cudaEventDestroy(ev);
    std::lock_guard<std::mutex> lk(g_tile_mu);
    g_tile_choice[{w, h}] = choice;
    return 0;  // `out` already holds the result
}

template <class S>
void launch_block_match(Plane<S, 4> img, Plane<S, 2> grad, Plane<S, 8> pca, const float* basis, Plane<S, 4> out,
                        const BlockMatchArgs& a, cudaStream_t s) {
    if constexpr (is_half<S>::value) {
        // the packed-FP32 matcher unless the call asks for the tensor-core one
        // (GLS_BM_TENSOR) or GLS_BM_KERNEL=mma selects it for the process
        static const bool mma_env = [] {
            const char* e = std::getenv("GLS_BM_KERNEL");
            return e && std::strcmp(e, "mma") == 0;
        }();
        if (a.tensor || mma_env) {
            launch_mma(img, grad, basis, out, a, s);
            return;
        }
        const int code = bm_tile_variant(img.w, img.h, [&](int c) {
            launch_pair_variant(c, img, grad, basis, out, a, s);
        }, s);
        if (code) launch_pair_variant(code, img, grad, basis, out, a, s);
    } else {
        ensure_dynamic_smem(reinterpret_cast<const void*>(k_block_match_plain<S>), int(sizeof(BmPlainSmem)));
        dim3 b(BP_TX, BP_TY);
        dim3 g((img.w + BP_TX - 1) / BP_TX, (img.h + 2 * BP_TY - 1) / (2 * BP_TY));
        k_block_match_plain<S><<<g, b, sizeof(BmPlainSmem), s>>>(img, grad, pca, out, a);
    }
}

template void launch_block_match<float>(Plane<float, 4>, Plane<float, 2>, Plane<float, 8>, const float*,
                                        Plane<float, 4>, const BlockMatchArgs&, cudaStream_t);
template void launch_block_match<__half>(Plane<__half, 4>, Plane<__half, 2>, Plane<__half, 8>, const float*,
                                         Plane<__half, 4>, const BlockMatchArgs&, cudaStream_t);

}  // namespace gls
