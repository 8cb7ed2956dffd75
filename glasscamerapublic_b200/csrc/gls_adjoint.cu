// gls_adjoint.cu — the hand-written adjoint of the pyramid denoise and
// reconstruct (PyramidProcessor<levels>::denoise, pyramid_processor.cpp:96-172,
// and the output transform, raw_converter.cpp:219) on the FP32 path.
//
// Given the forward's retained planes (per level: the layer that block
// matching denoised, its gradient plane, the denoised result, the frozen
// PCA basis) and dL/d(output RGB) of an MSE loss, it returns dL/dtheta for
// the per-level parameters that enter the pyramid:
//   luma_l, chroma_l       DenoiseParameters::luma / chroma (demosaic.hpp:33-40)
//   A_Y, B_Y, A_C, B_C     the level's YCbCr NLF a[0], b[0], a[1] = a[2], b[1] = b[2]
// The PCA basis is held fixed (its dependence on theta is not differentiated).
//
// Reverse sweep, fine to coarse: out = M den_0; den_l = BM_l(layer_l);
// layer_l = SN_l(img_l, img_{l+1}, den_{l+1}) for l < L-1, and
// layer_{L-1} = img_{L-1}. The pyramid parameters reach the loss through
// den_{l+1}; the raw green NLF reaches it through the input pyramid
// img_{l+1} = down(img_l), img_0 = the despeckled front-end output, so the
// sweep also accumulates dL/d img_l and pushes it down to img_0.
//   * k_adj_head          dL/d den_0 = M^T 2 (out - target) / N, and the loss
//   * k_bm_bwd_center     block matching, the pixel as the window centre:
//                         from the forward's outputs and kernel norms,
//                         recomputes its weights, then dL/d(its scales, its
//                         own PCA coefficients and chroma), dL/dtheta, and a
//                         per-pixel record for the neighbour pass
//   * k_bm_bwd_neighbor   the pixel as a neighbour q of every centre p whose
//                         window reads it (clamp-to-edge preimages included)
//   * k_pca_bwd           transpose of the 5x5 x 25x8 projection
//   * k_sn_bwd            subtractNoiseImage: dL/d(up-sampled den_{l+1}) and
//                         dL/dtheta through the sharpening gate
//   * k_up_bwd            transpose of the bilinear up-sampling (for the
//                         coarse denoised image, and with k_up_bwd_img for
//                         the coarse noisy image)
//   * k_down_bwd          transpose of the pyramid down-sampling: with the
//                         subtract-noise input terms, dL/d(level-0 image),
//                         which the raw front end's tangents
//                         (gls_front_jvp.cu) turn into dL/d(raw green NLF)
// Every reduction is per block and summed in block order: the gradient does
// not depend on scheduling.
#include <cfloat>

#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

constexpr int AT_X = 32, AT_Y = 8;        // adjoint tile (pixels)
constexpr int AH = 10;                     // block-matching window radius
constexpr int AW_ = AT_X + 2 * AH, AH_ = AT_Y + 2 * AH;

// offsets d in [-R, R] with clamp(p + d, 0, n - 1) == q
__device__ __forceinline__ bool preimage(int q, int p, int R, int n, int& lo, int& hi) {
    lo = q - p;
    hi = q - p;
    if (q == 0) lo = -R;
    if (q == n - 1) hi = R;
    lo = max(lo, -R);
    hi = min(hi, R);
    return lo <= hi;
}

__device__ __forceinline__ float sstep(float e0, float e1, float x, float* dx) {  // smoothstep and d/dx
    const float t = (x - e0) / (e1 - e0);
    if (t <= 0.f) {
        *dx = 0.f;
        return 0.f;
    }
    if (t >= 1.f) {
        *dx = 0.f;
        return 1.f;
    }
    *dx = 6.f * t * (1.f - t) / (e1 - e0);
    return t * t * (3.f - 2.f * t);
}

// Per-pixel scales of blockMatchingDenoiseImage (demosaic.metal:806-850)
// and their partial derivatives.
struct BmScales {
    float L, K1, K2;              // luma distance scale, chroma scales
    float dL_dsig0, dK1_dsig1, dK2_dsig2;
    float sig0, sig1, sig2;
};

__device__ __forceinline__ BmScales bm_scales(const AdjointLevelArgs& a, float y, float mag) {
    BmScales s;
    s.sig0 = sqrtf(a.var_a[0] + a.var_b[0] * y);
    s.sig1 = sqrtf(a.var_a[1] + a.var_b[1] * y);
    s.sig2 = sqrtf(a.var_a[2] + a.var_b[2] * y);
    const float dm0 = 1.f / (a.tm[0] * s.sig0), dm1 = 1.f / (a.tm[1] * s.sig1), dm2 = 1.f / (a.tm[2] * s.sig2);
    const float z = a.gradient_threshold * mag / s.sig0;
    float dedge_dz;
    const float edge = sstep(2.f, 16.f, z, &dedge_dz);
    const float den = 1.f + a.gradient_boost * edge;
    s.L = dm0 / den;
    // dL/dsig0 = -L / sig0 + dL/dedge * dedge/dz * dz/dsig0
    const float dL_dedge = -s.L * a.gradient_boost / den;
    s.dL_dsig0 = -s.L / s.sig0 + dL_dedge * dedge_dz * (-z / s.sig0);
    s.K1 = dm1 / a.chroma_boost;
    s.K2 = dm2 / a.chroma_boost;
    s.dK1_dsig1 = -s.K1 / s.sig1;
    s.dK2_dsig2 = -s.K2 / s.sig2;
    return s;
}

__device__ __forceinline__ float spatial_w(int i, int j) {
    const float d = 0.1f * sqrtf(float(i * i + j * j));
    return expf(-2.f * d * d);
}

struct CenterSmem {
    float4 q[AH_ * AW_][3];  // (Y, Cb, Cr, -), pca 0..3, pca 4..7 of the clamped window positions
    float sw[441];
};

// Block matching, the pixel p as the window centre. Writes the record
// (gY/ny, Y_out, gCb/nc, Cb_out, gCr/nc, Cr_out, L, K1, K2) the neighbour
// pass needs, the centre's own gradients (luma via its scales, chroma and
// PCA coefficients via the distances) and per-block dL/dtheta partials
// (luma, chroma, A_Y, B_Y, A_C, B_C).
__global__ void __launch_bounds__(256) k_bm_bwd_center(AdjointLevelArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CenterSmem& sm = *reinterpret_cast<CenterSmem*>(smem_raw);
    __shared__ float red[8][6];
    const int W = a.w, H = a.h;
    const int x0 = blockIdx.x * AT_X, y0 = blockIdx.y * AT_Y;
    const int tid = threadIdx.y * AT_X + threadIdx.x;
    for (int k = tid; k < 441; k += 256) sm.sw[k] = spatial_w(k % 21 - 10, k / 21 - 10);
    for (int k = tid; k < AH_ * AW_; k += 256) {
        const int ty = k / AW_, tx = k % AW_;
        const int sx = clampi(x0 - AH + tx, 0, W - 1), sy = clampi(y0 - AH + ty, 0, H - 1);
        const float4 l = *reinterpret_cast<const float4*>(a.layer + (size_t(sy) * W + sx) * 4);
        const float4* pc = reinterpret_cast<const float4*>(a.pca + (size_t(sy) * W + sx) * 8);
        sm.q[k][0] = make_float4(l.x, l.y, l.z, 0.f);
        sm.q[k][1] = pc[0];
        sm.q[k][2] = pc[1];
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    float th[6] = {0, 0, 0, 0, 0, 0};
    if (x < W && y < H) {
        const size_t pi = size_t(y) * W + x;
        const int c = (threadIdx.y + AH) * AW_ + threadIdx.x + AH;
        const float4 in = sm.q[c][0];
        const float4 ip0 = sm.q[c][1], ip1 = sm.q[c][2];
        const float ip[8] = {ip0.x, ip0.y, ip0.z, ip0.w, ip1.x, ip1.y, ip1.z, ip1.w};
        const float2 gr = *reinterpret_cast<const float2*>(a.grad + pi * 2);
        const float mag = sqrtf(gr.x * gr.x + gr.y * gr.y);
        const BmScales S = bm_scales(a, in.x, mag);
        const float L2 = S.L * S.L;
        // the forward's sums: outputs and the two kernel norms
        const float4 dv = *reinterpret_cast<const float4*>(a.den + pi * 4);
        const float Yo = dv.x, Cbo = dv.y, Cro = dv.z, ny = dv.w, nc = a.nc[pi];
        const float3 g = *reinterpret_cast<const float3*>(a.g_den + pi * 3);
        const float gYn = g.x / ny, gCbn = g.y / nc, gCrn = g.z / nc;
        // gradients of the centre's own quantities, tap by tap
        float gL = 0, gK1 = 0, gK2 = 0, gcb = 0, gcr = 0;
        float gip[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < 21; j++)
            for (int i = 0; i < 21; i++) {
                const int q = (threadIdx.y + j) * AW_ + threadIdx.x + i;
                const float4 s = sm.q[q][0], p0 = sm.q[q][1], p1 = sm.q[q][2];
                const float sp[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
                float d2 = 0.f;
#pragma unroll
                for (int k = 0; k < 8; k++) d2 += (sp[k] - ip[k]) * (sp[k] - ip[k]);
                const float lw = __expf(-2.f * d2 * L2);
                const float dcb = s.y - in.y, dcr = s.z - in.z;
                const float c1 = dcb * S.K1, c2 = dcr * S.K2;
                const float cw = __expf(-2.f * (lw * lw + c1 * c1 + c2 * c2));
                const float sw = sm.sw[j * 21 + i];
                const float gw = gYn * (s.x - Yo);
                const float gc = gCbn * (s.y - Cbo) + gCrn * (s.z - Cro);
                const float garg = -2.f * gc * sw * cw;
                const float glw = gw * sw + 2.f * garg * lw;
                const float gc1 = 2.f * garg * c1, gc2 = 2.f * garg * c2;
                const float gE = -2.f * glw * lw;  // E = d2 L^2
                gL += gE * 2.f * d2 * S.L;
                const float gd2 = gE * L2;
#pragma unroll
                for (int k = 0; k < 8; k++) gip[k] -= 2.f * gd2 * (sp[k] - ip[k]);
                gK1 += gc1 * dcb;
                gK2 += gc2 * dcr;
                gcb -= gc1 * S.K1;
                gcr -= gc2 * S.K2;
            }
        // scales -> centre luma and theta (ls = 1: no lens shading on this path)
        const float gsig0 = gL * S.dL_dsig0, gsig1 = gK1 * S.dK1_dsig1, gsig2 = gK2 * S.dK2_dsig2;
        const float gY = gsig0 * a.var_b[0] / (2.f * S.sig0) + gsig1 * a.var_b[1] / (2.f * S.sig1) +
                         gsig2 * a.var_b[2] / (2.f * S.sig2);
        th[0] = gL * (-S.L / a.tm[0]);                                     // luma
        th[1] = gK1 * (-S.K1 / a.tm[1]) + gK2 * (-S.K2 / a.tm[2]);        // chroma
        th[2] = gsig0 / (2.f * S.sig0);                                    // A_Y
        th[3] = gsig0 * in.x / (2.f * S.sig0);                             // B_Y
        th[4] = gsig1 / (2.f * S.sig1) + gsig2 / (2.f * S.sig2);           // A_C (a[1] = a[2])
        th[5] = (gsig1 / (2.f * S.sig1) + gsig2 / (2.f * S.sig2)) * in.x;  // B_C
        float* rec = a.rec + pi * 12;
        *reinterpret_cast<float4*>(rec) = make_float4(gYn, Yo, gCbn, Cbo);
        *reinterpret_cast<float4*>(rec + 4) = make_float4(gCrn, Cro, S.L, S.K1);
        *reinterpret_cast<float4*>(rec + 8) = make_float4(S.K2, 0.f, 0.f, 0.f);
        *reinterpret_cast<float4*>(a.g_layer + pi * 4) = make_float4(gY, gcb, gcr, 0.f);
        *reinterpret_cast<float4*>(a.g_pca + pi * 8) = make_float4(gip[0], gip[1], gip[2], gip[3]);
        *reinterpret_cast<float4*>(a.g_pca + pi * 8 + 4) = make_float4(gip[4], gip[5], gip[6], gip[7]);
    }
    // per-block theta partials, warp then block, fixed order
#pragma unroll
    for (int k = 0; k < 6; k++) {
        float v = th[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) red[tid >> 5][k] = v;
    }
    __syncthreads();
    if (tid < 6) {
        float v = 0.f;
        for (int w = 0; w < 8; w++) v += red[w][tid];
        a.part[(size_t(blockIdx.y) * gridDim.x + blockIdx.x) * 6 + tid] = v;
    }
}

// The neighbour pass stages 80 bytes per window position, so its tile is
// taller than the centre pass's: 32 x 16 pixels and 512 threads per block
// stage 52 x 36 positions (3.7 per pixel instead of 5.7) in 150 KB, and a
// block holds 16 warps on its SM.
constexpr int NT_Y = 16, NH_ = NT_Y + 2 * AH, NT_THREADS = AT_X * NT_Y;

struct NeighborSmem {
    float4 p[NH_ * AW_][5];  // (gYn, Yo, gCbn, Cbo), (gCrn, Cro, L, K1), (K2, cb, cr, -), pca 0..3, pca 4..7
    float sw[441];
};

// Block matching, the pixel q as a neighbour of every centre p whose
// window reads it (p in the 21 x 21 box around q; at the image border,
// every tap offset that clamps onto q).
__global__ void __launch_bounds__(NT_THREADS, 1) k_bm_bwd_neighbor(AdjointLevelArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    NeighborSmem& sm = *reinterpret_cast<NeighborSmem*>(smem_raw);
    const int W = a.w, H = a.h;
    const int x0 = blockIdx.x * AT_X, y0 = blockIdx.y * NT_Y;
    const int tid = threadIdx.y * AT_X + threadIdx.x;
    for (int k = tid; k < 441; k += NT_THREADS) sm.sw[k] = spatial_w(k % 21 - 10, k / 21 - 10);
    for (int k = tid; k < NH_ * AW_; k += NT_THREADS) {
        const int ty = k / AW_, tx = k % AW_;
        const int px = x0 - AH + tx, py = y0 - AH + ty;
        if (px < 0 || px >= W || py < 0 || py >= H) continue;  // not a pixel: never read
        const size_t pi = size_t(py) * W + px;
        const float* rec = a.rec + pi * 12;
        const float4 l = *reinterpret_cast<const float4*>(a.layer + pi * 4);
        sm.p[k][0] = *reinterpret_cast<const float4*>(rec);
        sm.p[k][1] = *reinterpret_cast<const float4*>(rec + 4);
        sm.p[k][2] = make_float4(rec[8], l.y, l.z, 0.f);
        sm.p[k][3] = *reinterpret_cast<const float4*>(a.pca + pi * 8);
        sm.p[k][4] = *reinterpret_cast<const float4*>(a.pca + pi * 8 + 4);
    }
    __syncthreads();
    const int qx = x0 + threadIdx.x, qy = y0 + threadIdx.y;
    if (qx >= W || qy >= H) return;
    const size_t qi = size_t(qy) * W + qx;
    const float4 s = *reinterpret_cast<const float4*>(a.layer + qi * 4);
    const float4 q0 = *reinterpret_cast<const float4*>(a.pca + qi * 8);
    const float4 q1 = *reinterpret_cast<const float4*>(a.pca + qi * 8 + 4);
    const float sp[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    float gs0 = 0, gs1 = 0, gs2 = 0;
    float gsp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // the contribution of centre p reading q through tap offset (i, j)
    auto pair = [&](int k, int ilo, int ihi, int jlo, int jhi) {
        const float4 r0 = sm.p[k][0], r1 = sm.p[k][1], r2 = sm.p[k][2], c0 = sm.p[k][3], c1v = sm.p[k][4];
        const float gYn = r0.x, Yo = r0.y, gCbn = r0.z, Cbo = r0.w;
        const float gCrn = r1.x, Cro = r1.y, L = r1.z, K1 = r1.w, K2 = r2.x, cbp = r2.y, crp = r2.z;
        const float ip[8] = {c0.x, c0.y, c0.z, c0.w, c1v.x, c1v.y, c1v.z, c1v.w};
        float d2 = 0.f;
#pragma unroll
        for (int m = 0; m < 8; m++) d2 += (sp[m] - ip[m]) * (sp[m] - ip[m]);
        const float L2 = L * L;
        const float lw = __expf(-2.f * d2 * L2);
        const float dcb = s.y - cbp, dcr = s.z - crp;
        const float c1 = dcb * K1, c2 = dcr * K2;
        const float cw = __expf(-2.f * (lw * lw + c1 * c1 + c2 * c2));
        const float gw = gYn * (s.x - Yo);
        const float gc = gCbn * (s.y - Cbo) + gCrn * (s.z - Cro);
        float gd2 = 0.f;
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                const float sw = sm.sw[(j + AH) * 21 + i + AH];
                const float wy = sw * lw, wc = sw * cw;
                const float garg = -2.f * gc * sw * cw;
                const float glw = gw * sw + 2.f * garg * lw;
                gs0 += gYn * wy;
                gs1 += gCbn * wc + 2.f * garg * c1 * K1;
                gs2 += gCrn * wc + 2.f * garg * c2 * K2;
                gd2 += -2.f * glw * lw * L2;
            }
#pragma unroll
        for (int m = 0; m < 8; m++) gsp[m] += 2.f * gd2 * (sp[m] - ip[m]);
    };
    const int py0 = max(qy - AH, 0), py1 = min(qy + AH, H - 1);
    const int px0 = max(qx - AH, 0), px1 = min(qx + AH, W - 1);
    if (qx > 0 && qx < W - 1 && qy > 0 && qy < H - 1) {
        // not on the image border: every centre reads q through exactly one tap
        for (int py = py0; py <= py1; py++) {
            const int j = qy - py;
            for (int px = px0; px <= px1; px++) {
                const int i = qx - px;
                pair((py - y0 + AH) * AW_ + (px - x0 + AH), i, i, j, j);
            }
        }
    } else {
        for (int py = py0; py <= py1; py++) {
            int jlo, jhi;
            if (!preimage(qy, py, AH, H, jlo, jhi)) continue;
            for (int px = px0; px <= px1; px++) {
                int ilo, ihi;
                if (!preimage(qx, px, AH, W, ilo, ihi)) continue;
                pair((py - y0 + AH) * AW_ + (px - x0 + AH), ilo, ihi, jlo, jhi);
            }
        }
    }
    float4* gl = reinterpret_cast<float4*>(a.g_layer + qi * 4);
    const float4 cur = *gl;
    *gl = make_float4(cur.x + gs0, cur.y + gs1, cur.z + gs2, 0.f);
    float4* gp = reinterpret_cast<float4*>(a.g_pca + qi * 8);
    const float4 p0 = gp[0], p1 = gp[1];
    gp[0] = make_float4(p0.x + gsp[0], p0.y + gsp[1], p0.z + gsp[2], p0.w + gsp[3]);
    gp[1] = make_float4(p1.x + gsp[4], p1.y + gsp[5], p1.z + gsp[6], p1.w + gsp[7]);
}

// pcaProjection transposed (demosaic.metal:774-796): dL/d luma(x) +=
// sum over the patches that read x of basis . dL/d pca.
__global__ void __launch_bounds__(256) k_pca_bwd(AdjointLevelArgs a) {
    __shared__ float B[25][8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < 200) B[tid / 8][tid % 8] = a.basis[tid];
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    float acc = 0.f;
    for (int py = max(y - 2, 0); py <= min(y + 2, a.h - 1); py++) {
        int jlo, jhi;
        if (!preimage(y, py, 2, a.h, jlo, jhi)) continue;
        for (int px = max(x - 2, 0); px <= min(x + 2, a.w - 1); px++) {
            int ilo, ihi;
            if (!preimage(x, px, 2, a.w, ilo, ihi)) continue;
            const float* gp = a.g_pca + (size_t(py) * a.w + px) * 8;
            float g[8];
#pragma unroll
            for (int m = 0; m < 8; m++) g[m] = gp[m];
            for (int j = jlo; j <= jhi; j++)
                for (int i = ilo; i <= ihi; i++) {
                    const int row = (j + 2) * 5 + (i + 2);
#pragma unroll
                    for (int m = 0; m < 8; m++) acc += B[row][m] * g[m];
                }
        }
    }
    a.g_layer[(size_t(y) * a.w + x) * 4] += acc;
}

// 2 (out - target) / N through the output transform; the loss per block.
__global__ void __launch_bounds__(256) k_adj_head(const float* __restrict__ den0, const float* __restrict__ target,
                                                  int tstride, int w, int h, AdjointHeadArgs a,
                                                  float* __restrict__ g_den, double* __restrict__ loss_part) {
    __shared__ double red[8];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (x < w && y < h) {
        const size_t pi = size_t(y) * w + x;
        const float4 d = *reinterpret_cast<const float4*>(den0 + pi * 4);
        const float v[3] = {d.x, d.y, d.z};
        float go[3];
        const float* t = target + pi * tstride;
        for (int r = 0; r < 3; r++) {
            const float o = a.m[r * 3 + 0] * v[0] + a.m[r * 3 + 1] * v[1] + a.m[r * 3 + 2] * v[2];
            const float e = o - t[r];
            l += double(e) * double(e);
            go[r] = 2.f * e * a.inv_n;
        }
        float gd[3];
        for (int c = 0; c < 3; c++) gd[c] = a.m[0 * 3 + c] * go[0] + a.m[1 * 3 + c] * go[1] + a.m[2 * 3 + c] * go[2];
        g_den[pi * 3 + 0] = gd[0];
        g_den[pi * 3 + 1] = gd[1];
        g_den[pi * 3 + 2] = gd[2];
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((tid & 31) == 0) red[tid >> 5] = l;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
        for (int k = 0; k < 8; k++) s += red[k];
        loss_part[size_t(blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// subtractNoiseImage (demosaic.metal:922-959) transposed with respect to
// the up-sampled denoised coarse level (per fine pixel, 3 channels) and to
// the gate's noise model (nlf_a = A_Y luma, nlf_b = B_Y luma).
__global__ void __launch_bounds__(256) k_sn_bwd(AdjointSnArgs a) {
    __shared__ float red[8][2];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    float gna = 0.f, gnb = 0.f;
    if (x < a.w && y < a.h) {
        const size_t pi = size_t(y) * a.w + x;
        const float u = (float(x) + 0.5f) * a.rx - 0.5f, v = (float(y) + 0.5f) * a.ry - 0.5f;
        const float fu = floorf(u), fv = floorf(v);
        const int xi = int(fu), yi = int(fv);
        const float ax = u - fu, ay = v - fv;
        auto bil = [&](const float* p, int c) {
            auto at = [&](int X, int Y) {
                X = clampi(X, 0, a.cw - 1);
                Y = clampi(Y, 0, a.ch - 1);
                return p[(size_t(Y) * a.cw + X) * 4 + c];
            };
            const float A = at(xi, yi), Bv = at(xi + 1, yi), Cv = at(xi, yi + 1), D = at(xi + 1, yi + 1);
            const float top = A + (Bv - A) * ax, bot = Cv + (D - Cv) * ax;
            return top + (bot - top) * ay;
        };
        const float4 ip = *reinterpret_cast<const float4*>(a.in + pi * 4);
        const float ipv[3] = {ip.x, ip.y, ip.z};
        float p1[3], pd[3], dn[3];
        for (int c = 0; c < 3; c++) {
            p1[c] = bil(a.coarse, c);
            pd[c] = bil(a.coarse_den, c);
            dn[c] = ipv[c] - (c == 0 ? a.luma_weight : 1.f) * (p1[c] - pd[c]);
        }
        float alpha = a.sharpening, dalpha_dpd0 = 0.f, dalpha_dna = 0.f, dalpha_dnb = 0.f;
        if (a.sharpening > 1.f) {
            const float2 g = *reinterpret_cast<const float2*>(a.grad + pi * 2);
            const float gm = sqrtf(g.x * g.x + g.y * g.y);
            const float sigma = sqrtf(a.nlf_a + a.nlf_b * pd[0]);
            // S1 = smoothstep(sigma, 4 sigma, gm): t = gm / (3 sigma) - 1/3
            float dS1_dt;
            const float S1 = sstep(0.f, 1.f, gm / (3.f * sigma) - 1.f / 3.f, &dS1_dt);
            const float dS1_dsig = dS1_dt * (-gm / (3.f * sigma * sigma));
            float dS2, dS3;
            const float S2 = sstep(0.75f, 0.95f, pd[0], &dS2), S3 = sstep(0.05f, 0.1f, pd[0], &dS3);
            const float detail = S1 * (1.f - S2) * S3;
            alpha = 1.f + (a.sharpening - 1.f) * detail;
            const float k = a.sharpening - 1.f;
            const float ddet_dsig = dS1_dsig * (1.f - S2) * S3;
            dalpha_dpd0 = k * (ddet_dsig * a.nlf_b / (2.f * sigma) - S1 * dS2 * S3 + S1 * (1.f - S2) * dS3);
            dalpha_dna = k * ddet_dsig / (2.f * sigma);
            dalpha_dnb = k * ddet_dsig * pd[0] / (2.f * sigma);
        }
        const float4 go4 = *reinterpret_cast<const float4*>(a.g_layer + pi * 4);
        float go[3] = {go4.x, go4.y, go4.z};
        const float o0 = pd[0] + (dn[0] - pd[0]) * alpha;
        if (!(o0 > 0.f)) go[0] = 0.f;  // max(o, 0)
        float galpha = 0.f, gpd[3];
        for (int c = 0; c < 3; c++) {
            const float wc = c == 0 ? a.luma_weight : 1.f;
            galpha += go[c] * (dn[c] - pd[c]);
            gpd[c] = go[c] * (1.f - alpha + alpha * wc);
        }
        gpd[0] += galpha * dalpha_dpd0;
        gna = galpha * dalpha_dna;
        gnb = galpha * dalpha_dnb;
        a.g_up[pi * 3 + 0] = gpd[0];
        a.g_up[pi * 3 + 1] = gpd[1];
        a.g_up[pi * 3 + 2] = gpd[2];
        if (a.g_in) {  // d(out)/d(in) = alpha, d(out)/d(up-sampled coarse) = -alpha * weight
            for (int c = 0; c < 3; c++) {
                const float wc = c == 0 ? a.luma_weight : 1.f;
                a.g_in[pi * 3 + c] += alpha * go[c];
                a.g_p1[pi * 3 + c] = -alpha * wc * go[c];
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        gna += __shfl_down_sync(0xffffffffu, gna, o);
        gnb += __shfl_down_sync(0xffffffffu, gnb, o);
    }
    if ((tid & 31) == 0) {
        red[tid >> 5][0] = gna;
        red[tid >> 5][1] = gnb;
    }
    __syncthreads();
    if (tid < 2) {
        float v = 0.f;
        for (int w = 0; w < 8; w++) v += red[w][tid];
        a.part[(size_t(blockIdx.y) * gridDim.x + blockIdx.x) * 2 + tid] = v;
    }
}

// bilinear up-sampling (the reconstruct step's coarse reads) transposed:
// each coarse pixel gathers the weights with which fine pixels sampled it.
__device__ __forceinline__ void up_transpose(const AdjointSnArgs& a, const float* src, float* dst, bool accumulate) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= a.cw || Y >= a.ch) return;
    float acc[3] = {0, 0, 0};
    for (int y = max(2 * Y - 4, 0); y <= min(2 * Y + 4, a.h - 1); y++) {
        const float v = (float(y) + 0.5f) * a.ry - 0.5f;
        const float fv = floorf(v);
        const int yi = int(fv);
        const float ay = v - fv;
        const float wy = (clampi(yi, 0, a.ch - 1) == Y ? 1.f - ay : 0.f) + (clampi(yi + 1, 0, a.ch - 1) == Y ? ay : 0.f);
        if (wy == 0.f) continue;
        for (int x = max(2 * X - 4, 0); x <= min(2 * X + 4, a.w - 1); x++) {
            const float u = (float(x) + 0.5f) * a.rx - 0.5f;
            const float fu = floorf(u);
            const int xi = int(fu);
            const float ax = u - fu;
            const float wx =
                (clampi(xi, 0, a.cw - 1) == X ? 1.f - ax : 0.f) + (clampi(xi + 1, 0, a.cw - 1) == X ? ax : 0.f);
            if (wx == 0.f) continue;
            const float* g = src + (size_t(y) * a.w + x) * 3;
            const float wgt = wx * wy;
            acc[0] += wgt * g[0];
            acc[1] += wgt * g[1];
            acc[2] += wgt * g[2];
        }
    }
    float* o = dst + (size_t(Y) * a.cw + X) * 3;
    for (int c = 0; c < 3; c++) o[c] = accumulate ? o[c] + acc[c] : acc[c];
}

__global__ void __launch_bounds__(256) k_up_bwd(AdjointSnArgs a) { up_transpose(a, a.g_up, a.g_coarse_den, false); }
__global__ void __launch_bounds__(256) k_up_bwd_img(AdjointSnArgs a) { up_transpose(a, a.g_p1, a.g_coarse_img, true); }

// k_downsample transposed: out(x, y) = 1/4 sum over a, b in {0, 1} of the
// bilinear sample at (x rx - 0.5 + a rx, y ry - 0.5 + b ry), clamp-to-edge,
// a separable weight; each fine pixel gathers from the coarse pixels whose
// samples touch it.
__device__ __forceinline__ float down_weight(int X, int x, float r, int n) {
    float wsum = 0.f;
    for (int t = 0; t < 2; t++) {
        const float u = __fsub_rn(__fmul_rn(float(x + t), r), 0.5f);
        const float fu = floorf(u);
        const int xi = int(fu);
        const float ax = u - fu;
        wsum += (clampi(xi, 0, n - 1) == X ? 1.f - ax : 0.f) + (clampi(xi + 1, 0, n - 1) == X ? ax : 0.f);
    }
    return wsum;
}

__global__ void __launch_bounds__(256) k_down_bwd(const float* __restrict__ gc, int cw, int ch, float* __restrict__ gf,
                                                 int w, int h, float rx, float ry) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
    if (X >= w || Y >= h) return;
    const int x0 = max(int(floorf(float(X) / rx)) - 3, 0), x1 = min(int(floorf(float(X) / rx)) + 3, cw - 1);
    const int y0 = max(int(floorf(float(Y) / ry)) - 3, 0), y1 = min(int(floorf(float(Y) / ry)) + 3, ch - 1);
    float acc[3] = {0, 0, 0};
    for (int y = y0; y <= y1; y++) {
        const float wy = down_weight(Y, y, ry, h);
        if (wy == 0.f) continue;
        for (int x = x0; x <= x1; x++) {
            const float wx = down_weight(X, x, rx, w);
            if (wx == 0.f) continue;
            const float wgt = 0.25f * wx * wy;
            const float* g = gc + (size_t(y) * cw + x) * 3;
            acc[0] += wgt * g[0];
            acc[1] += wgt * g[1];
            acc[2] += wgt * g[2];
        }
    }
    float* o = gf + (size_t(Y) * w + X) * 3;
    o[0] += acc[0];
    o[1] += acc[1];
    o[2] += acc[2];
}

__global__ void __launch_bounds__(256) k_add_layer_grad(const float* __restrict__ gl, float* __restrict__ gi, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int c = 0; c < 3; c++) gi[size_t(i) * 3 + c] += gl[size_t(i) * 4 + c];
}

// 3-channel gradient planes to and from caller views of 3 or 4 channels
__global__ void __launch_bounds__(256) k_pack3(const float* __restrict__ src, size_t pitch, int ch,
                                              float* __restrict__ dst, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float* p = src + size_t(y) * pitch + size_t(x) * ch;
    float* o = dst + (size_t(y) * w + x) * 3;
    o[0] = p[0];
    o[1] = p[1];
    o[2] = p[2];
}

__global__ void __launch_bounds__(256) k_unpack3(const float* __restrict__ src, float* __restrict__ dst, size_t pitch,
                                                int ch, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float* p = src + (size_t(y) * w + x) * 3;
    float* o = dst + size_t(y) * pitch + size_t(x) * ch;
    o[0] = p[0];
    o[1] = p[1];
    o[2] = p[2];
    if (ch == 4) o[3] = 0.f;
}

void launch_pack3(const float* src, size_t pitch_floats, int channels, float* dst, int w, int h, cudaStream_t s) {
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    k_pack3<<<g, b, 0, s>>>(src, pitch_floats, channels, dst, w, h);
}

void launch_unpack3(const float* src, float* dst, size_t pitch_floats, int channels, int w, int h, cudaStream_t s) {
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    k_unpack3<<<g, b, 0, s>>>(src, dst, pitch_floats, channels, w, h);
}

size_t adjoint_center_smem() { return sizeof(CenterSmem); }
size_t adjoint_neighbor_smem() { return sizeof(NeighborSmem); }

void launch_adj_head(const float* den0, const float* target, int tstride, int w, int h, const AdjointHeadArgs& a,
                     float* g_den, double* loss_part, cudaStream_t s) {
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    k_adj_head<<<g, b, 0, s>>>(den0, target, tstride, w, h, a, g_den, loss_part);
}

void launch_bm_bwd(const AdjointLevelArgs& a, cudaStream_t s) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_bm_bwd_center), int(sizeof(CenterSmem)));
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_bm_bwd_neighbor), int(sizeof(NeighborSmem)));
    const dim3 b(AT_X, AT_Y), g((a.w + AT_X - 1) / AT_X, (a.h + AT_Y - 1) / AT_Y);
    k_bm_bwd_center<<<g, b, sizeof(CenterSmem), s>>>(a);
    const dim3 nb(AT_X, NT_Y), ng((a.w + AT_X - 1) / AT_X, (a.h + NT_Y - 1) / NT_Y);
    k_bm_bwd_neighbor<<<ng, nb, sizeof(NeighborSmem), s>>>(a);
    const dim3 b2(32, 8), g2((a.w + 31) / 32, (a.h + 7) / 8);
    k_pca_bwd<<<g2, b2, 0, s>>>(a);
}

void launch_sn_bwd(const AdjointSnArgs& a, cudaStream_t s) {
    const dim3 b(32, 8), g((a.w + 31) / 32, (a.h + 7) / 8), gc((a.cw + 31) / 32, (a.ch + 7) / 8);
    k_sn_bwd<<<g, b, 0, s>>>(a);
    k_up_bwd<<<gc, b, 0, s>>>(a);
    if (a.g_in) k_up_bwd_img<<<gc, b, 0, s>>>(a);
}

void launch_add_layer_grad(const float* g_layer, float* g_img, int w, int h, cudaStream_t s) {
    const int n = w * h;
    k_add_layer_grad<<<(n + 255) / 256, 256, 0, s>>>(g_layer, g_img, n);
}

void launch_down_bwd(const float* g_coarse, int cw, int ch, float* g_fine, int w, int h, cudaStream_t s) {
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    k_down_bwd<<<g, b, 0, s>>>(g_coarse, cw, ch, g_fine, w, h, float(w) / float(cw), float(h) / float(ch));
}

int adjoint_blocks(int w, int h) { return ((w + AT_X - 1) / AT_X) * ((h + AT_Y - 1) / AT_Y); }
int adjoint_sn_blocks(int w, int h) { return ((w + 31) / 32) * ((h + 7) / 8); }

}  // namespace gls
