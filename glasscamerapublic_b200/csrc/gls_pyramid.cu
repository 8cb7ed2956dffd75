// gls_pyramid.cu — kernels of PyramidProcessor<levels>::denoise
// (pyramid_processor.cpp:96-172): Gaussian-pyramid downsample, the
// reconstruct (noise subtraction) step, the per-level PCA patch basis
// (covariance + FP64 Jacobi eigen-solve on the device), the 5x5-patch PCA
// projection and the 21x21 block-matching non-local-means denoise.
#include <cmath>
#include <cstdio>

#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

// --------------------------------------------------------------------------
// downsampleImageXYZ / downsampleImageXY, demosaic.metal:886-920: mean of
// four bilinear samples at texel-space (x*r - 0.5, (x+1)*r - 0.5) with
// r = in/out size (a 4x4 box for an exact halving). Positions are formed
// with explicit FP32 roundings, matching the oracle's FP32 run.
template <class S, int C>
__global__ void __launch_bounds__(256) k_downsample(Plane<S, C> in, Plane<S, C> out, float rx, float ry) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out.w || y >= out.h) return;
    const float u[2] = {__fsub_rn(__fmul_rn(float(x), rx), 0.5f), __fsub_rn(__fmul_rn(float(x + 1), rx), 0.5f)};
    const float v[2] = {__fsub_rn(__fmul_rn(float(y), ry), 0.5f), __fsub_rn(__fmul_rn(float(y + 1), ry), 0.5f)};
    float acc[C > 2 ? 3 : 2] = {};
    constexpr int NC = C > 2 ? 3 : 2;
#pragma unroll
    for (int b = 0; b < 2; b++)
#pragma unroll
        for (int a = 0; a < 2; a++) {
            const float fu = floorf(u[a]), fv = floorf(v[b]);
            const int xi = int(fu), yi = int(fv);
            const float ax = u[a] - fu, ay = v[b] - fv;
            float t00[4], t01[4], t10[4], t11[4];
            auto ld = [&](int xx, int yy, float* dst) {
                const S* p = in.pxc(xx, yy);
                if constexpr (C == 4) {
                    const f4 q = ld4<S>(p);
                    dst[0] = q.x; dst[1] = q.y; dst[2] = q.z;
                } else {
                    const f2 q = ld2<S>(p);
                    dst[0] = q.x; dst[1] = q.y;
                }
            };
            ld(xi, yi, t00);
            ld(xi + 1, yi, t01);
            ld(xi, yi + 1, t10);
            ld(xi + 1, yi + 1, t11);
#pragma unroll
            for (int c = 0; c < NC; c++) {
                const float top = t00[c] + (t01[c] - t00[c]) * ax;
                const float bot = t10[c] + (t11[c] - t10[c]) * ax;
                acc[c] += top + (bot - top) * ay;
            }
        }
    if constexpr (C == 4) {
        st4<S>(out.px(x, y), f4{0.25f * acc[0], 0.25f * acc[1], 0.25f * acc[2], 0.f});
    } else {
        st2<S>(out.px(x, y), f2{0.25f * acc[0], 0.25f * acc[1]});
    }
}

// --------------------------------------------------------------------------
// subtractNoiseImage, demosaic.metal:922-959: subtract the coarse level's
// removed noise (bilinear up-sampled) and apply the noise-gated sharpening.
template <class S>
__device__ __forceinline__ void bilin3(const Plane<S, 4>& p, float u, float v, float out[3]) {
    const float fu = floorf(u), fv = floorf(v);
    const int xi = int(fu), yi = int(fv);
    const float ax = u - fu, ay = v - fv;
    const f4 a = ld4<S>(p.pxc(xi, yi)), b = ld4<S>(p.pxc(xi + 1, yi));
    const f4 c = ld4<S>(p.pxc(xi, yi + 1)), d = ld4<S>(p.pxc(xi + 1, yi + 1));
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z}, cv[3] = {c.x, c.y, c.z}, dv[3] = {d.x, d.y, d.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const float top = av[k] + (bv[k] - av[k]) * ax;
        const float bot = cv[k] + (dv[k] - cv[k]) * ax;
        out[k] = top + (bot - top) * ay;
    }
}

template <class S>
__global__ void __launch_bounds__(256) k_subtract_noise(Plane<S, 4> in, Plane<S, 4> coarse, Plane<S, 4> coarse_den,
                                                        Plane<S, 2> grad, Plane<S, 4> out, SubtractArgs a, float rx,
                                                        float ry) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= in.w || y >= in.h) return;
    const float u = __fsub_rn(__fmul_rn(__fadd_rn(float(x), 0.5f), rx), 0.5f);
    const float v = __fsub_rn(__fmul_rn(__fadd_rn(float(y), 0.5f), ry), 0.5f);
    const f4 ip = ld4<S>(in.px(x, y));
    float p1[3], pd[3];
    bilin3(coarse, u, v, p1);
    bilin3(coarse_den, u, v, pd);
    const float ipv[3] = {ip.x, ip.y, ip.z};
    float dn[3];
#pragma unroll
    for (int c = 0; c < 3; c++) dn[c] = ipv[c] - (c == 0 ? a.luma_weight : 1.f) * (p1[c] - pd[c]);
    float alpha = a.sharpening;
    if (a.sharpening > 1.f) {
        const f2 g = ld2<S>(grad.px(x, y));
        const float gm = sqrtf(g.x * g.x + g.y * g.y);
        const float sigma = sqrtf(a.nlf_a + a.nlf_b * pd[0]);
        const float detail = smoothstepf(sigma, 4.f * sigma, gm) * (1.f - smoothstepf(0.75f, 0.95f, pd[0])) *
                             smoothstepf(0.05f, 0.1f, pd[0]);
        alpha = 1.f + (alpha - 1.f) * detail;
    }
    f4 o;
    o.x = fmaxf(mixf(pd[0], dn[0], alpha), 0.f);
    o.y = mixf(pd[1], dn[1], alpha);
    o.z = mixf(pd[2], dn[2], alpha);
    o.w = ip.w;
    st4<S>(out.px(x, y), o);
}

// --------------------------------------------------------------------------
// PCA patch covariance: collectPatches (demosaic.metal:755-772) fused with
// the covariance reduction of build_pca_space (PCA.cpp:29-33). Patches are
// the 5x5 luma neighbourhoods of (8x, 8y), x < W/8, y < H/8. Each block
// stages 64 patches in shared memory; thread t < 325 owns one upper-triangle
// entry of sum p p^T and thread 325 + r the sum of component r, in FP64.
// Each block writes its partial sums to its own row of `part`; the rows are
// summed in block order afterwards, so the result does not depend on
// scheduling (no atomics).
__constant__ uint8_t kPairR[325], kPairC[325];

constexpr int PC_CHUNK = 64;

template <class S>
__global__ void __launch_bounds__(352) k_pca_cov(Plane<S, 4> img, double* __restrict__ part) {
    __shared__ float sp[PC_CHUNK][kPcaDim + 1];
    const int gw = img.w / 8, gh = img.h / 8;
    const int n = gw * gh;
    const int t = threadIdx.x;
    double sum = 0.0;
    int r = 0, c = 0;
    if (t < 325) {
        r = kPairR[t];
        c = kPairC[t];
    } else if (t < 350) {
        r = t - 325;
    }
    for (int base = blockIdx.x * PC_CHUNK; base < n; base += gridDim.x * PC_CHUNK) {
        const int cnt = min(PC_CHUNK, n - base);
        for (int i = t; i < cnt * kPcaDim; i += blockDim.x) {
            const int k = i / kPcaDim, e = i % kPcaDim;
            const int pidx = base + k;
            const int px = (pidx % gw) * 8 + (e % 5) - 2, py = (pidx / gw) * 8 + (e / 5) - 2;
            sp[k][e] = to_f(*img.pxc(px, py));
        }
        __syncthreads();
        if (t < 325) {
            for (int k = 0; k < cnt; k++) sum += double(sp[k][r]) * double(sp[k][c]);
        } else if (t < 350) {
            for (int k = 0; k < cnt; k++) sum += double(sp[k][r]);
        }
        __syncthreads();
    }
    if (t < 350) part[blockIdx.x * kPcaAcc + t] = sum;
}

// --------------------------------------------------------------------------
// Symmetric eigen-solve of the 25x25 patch covariance (replaces Eigen's
// SelfAdjointEigenSolver, PCA.cpp:36): parallel cyclic Jacobi in FP64 on a
// 26x26 matrix (25 + one zero pad row/column) with the round-robin pair
// schedule (13 disjoint rotations per round, 25 rounds per sweep). One
// block of 1024 threads; every sweep is a bounded loop (at most 40 sweeps),
// so the kernel always ends. The top-8 eigenvectors (descending eigenvalue,
// each signed so its largest-magnitude entry is positive) are written as a
// row-major 25x8 FP32 basis. status receives the sweep count, or -1 when
// the sweep limit was hit before convergence.
constexpr int EJ_N = 26;

__global__ void __launch_bounds__(1024) k_pca_eigen(const double* __restrict__ part, int n_blocks, int n_patches,
                                                   float* __restrict__ basis, int* status) {
    __shared__ double acc[kPcaAcc];
    __shared__ double A[EJ_N][EJ_N + 1], B[EJ_N][EJ_N + 1], V[EJ_N][EJ_N + 1], V2[EJ_N][EJ_N + 1];
    __shared__ double rc[EJ_N], rs[EJ_N];  // per index: rotation (c, s)
    __shared__ int partner[EJ_N], isp[EJ_N];
    __shared__ double red[32];
    __shared__ int done, order[25];
    const int t = threadIdx.x;
    const int i = t / EJ_N, j = t % EJ_N;
    const bool act = t < EJ_N * EJ_N;

    if (n_patches < 2) {
        if (t < 25 * 8) basis[t] = ((t / 8) == (t % 8)) ? 1.f : 0.f;
        if (t == 0 && status) *status = 0;
        return;
    }
    // block partials summed in block order (deterministic)
    if (t < kPcaAcc) {
        double v = 0.0;
        for (int b = 0; b < n_blocks; b++) v += part[b * kPcaAcc + t];
        acc[t] = v;
    }
    __syncthreads();
    // covariance from raw moments
    if (act) {
        double v = 0.0;
        if (i < 25 && j < 25) {
            const int r = min(i, j), c = max(i, j);
            const int idx = r * 25 - r * (r - 1) / 2 + (c - r);  // upper-triangle index (row-major)
            const double n = double(n_patches);
            const double mi = acc[325 + i] / n, mj = acc[325 + j] / n;
            v = (acc[idx] - n * mi * mj) / (n - 1.0);
        }
        A[i][j] = v;
        V[i][j] = (i == j) ? 1.0 : 0.0;
    }
    if (t == 0) done = 0;
    __syncthreads();

    int sweep = 0;
    for (; sweep < 40; sweep++) {
        // convergence test: off-diagonal vs total Frobenius mass
        double off = 0.0, tot = 0.0;
        if (act) {
            const double a = A[i][j];
            tot = a * a;
            off = (i != j) ? a * a : 0.0;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_down_sync(0xffffffffu, off, o);
            tot += __shfl_down_sync(0xffffffffu, tot, o);
        }
        __shared__ double red2[32];
        if ((t & 31) == 0) {
            red[t >> 5] = off;
            red2[t >> 5] = tot;
        }
        __syncthreads();
        if (t == 0) {
            double so = 0, st = 0;
            for (int k = 0; k < 32; k++) {
                so += red[k];
                st += red2[k];
            }
            done = (so <= 1e-26 * st || so == 0.0) ? 1 : 0;  // off-diagonal norm <= 1e-13 x total
        }
        __syncthreads();
        if (done) break;
        for (int round = 0; round < 25; round++) {
            // pairs of this round: (25, round) and ((round+m)%25, (round-m+25)%25), m = 1..12
            if (t < 13) {
                int p, q;
                if (t == 0) {
                    p = round;
                    q = 25;
                } else {
                    p = (round + t) % 25;
                    q = (round - t + 25) % 25;
                }
                if (p > q) {
                    const int tmp = p;
                    p = q;
                    q = tmp;
                }
                const double apq = A[p][q], app = A[p][p], aqq = A[q][q];
                double c = 1.0, s = 0.0;
                if (fabs(apq) >= 1e-300) {
                    const double theta = (aqq - app) / (2.0 * apq);
                    const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(tt * tt + 1.0);
                    s = tt * c;
                }
                rc[p] = c; rs[p] = s; partner[p] = q; isp[p] = 1;
                rc[q] = c; rs[q] = s; partner[q] = p; isp[q] = 0;
            }
            __syncthreads();
            // columns: B = A J, V2 = V J
            if (act) {
                const int pj = partner[j];
                const double c = rc[j], s = rs[j];
                if (isp[j]) {
                    B[i][j] = c * A[i][j] - s * A[i][pj];
                    V2[i][j] = c * V[i][j] - s * V[i][pj];
                } else {
                    B[i][j] = s * A[i][pj] + c * A[i][j];
                    V2[i][j] = s * V[i][pj] + c * V[i][j];
                }
            }
            __syncthreads();
            // rows: A = J^T B
            if (act) {
                const int pi = partner[i];
                const double c = rc[i], s = rs[i];
                if (isp[i]) A[i][j] = c * B[i][j] - s * B[pi][j];
                else A[i][j] = s * B[pi][j] + c * B[i][j];
                V[i][j] = V2[i][j];
            }
            __syncthreads();
        }
    }
    // order eigenvalues descending (stable by index)
    if (t == 0) {
        for (int k = 0; k < 25; k++) order[k] = k;
        for (int k = 1; k < 25; k++) {  // insertion sort, stable
            const int e = order[k];
            int m = k - 1;
            while (m >= 0 && A[order[m]][order[m]] < A[e][e]) {
                order[m + 1] = order[m];
                m--;
            }
            order[m + 1] = e;
        }
        if (status) *status = sweep < 40 ? sweep : -1;
    }
    __syncthreads();
    // sorted eigenpairs into B (column c = c-th largest), then the top-8 basis
    __shared__ double ev[25], work[200];
    if (t < 25) ev[t] = A[order[t]][order[t]];
    if (t < 625) B[t / 25][t % 25] = V[t / 25][order[t % 25]];
    __syncthreads();
    if (t == 0) select_pca_basis(ev, &B[0][0], EJ_N + 1, work, basis);
}

// --------------------------------------------------------------------------
// pcaProjection, demosaic.metal:774-796: 5x5 luma patch times the 25x8
// basis -> 8 coefficients per pixel.
template <class S>
__global__ void __launch_bounds__(256) k_pca_project(Plane<S, 4> img, const float* __restrict__ basis,
                                                     Plane<S, 8> out) {
    __shared__ float b[25][8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < 200) b[tid / 8][tid % 8] = basis[tid];
    __syncthreads();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= img.w || y >= img.h) return;
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int row = 0;
#pragma unroll
    for (int j = -2; j <= 2; j++)
#pragma unroll
        for (int i = -2; i <= 2; i++, row++) {
            const float v = to_f(*img.pxc(x + i, y + j));
#pragma unroll
            for (int c = 0; c < 8; c++) acc[c] += b[row][c] * v;
        }
    S* o = out.px(x, y);
    if constexpr (is_half<S>::value) {
        uint4 u;
        __half2 h0 = __floats2half2_rn(acc[0], acc[1]), h1 = __floats2half2_rn(acc[2], acc[3]);
        __half2 h2 = __floats2half2_rn(acc[4], acc[5]), h3 = __floats2half2_rn(acc[6], acc[7]);
        u.x = *reinterpret_cast<uint32_t*>(&h0);
        u.y = *reinterpret_cast<uint32_t*>(&h1);
        u.z = *reinterpret_cast<uint32_t*>(&h2);
        u.w = *reinterpret_cast<uint32_t*>(&h3);
        *reinterpret_cast<uint4*>(o) = u;
    } else {
        float4* o4 = reinterpret_cast<float4*>(o);
        o4[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        o4[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
    }
}

// --------------------------------------------------------------------------
// blockMatchingDenoiseImage, demosaic.metal:806-884. Output tile 16 x 16,
// one pixel per thread; the tile's 36 x 36 window region of YCbCr and PCA
// coefficients is staged in shared memory (FP32), the spatial Gaussian
// gaussian(0.1 |(i, j)|) is a 21 x 21 table.
constexpr int BM_T = 16, BM_R = 10, BM_W = BM_T + 2 * BM_R;

struct BlockMatchSmem {
    float4 pca[BM_W * BM_W][2];
    float4 ycc[BM_W * BM_W];
    float spatial[21 * 21];
};

template <class S>
__global__ void __launch_bounds__(256) k_block_match(Plane<S, 4> img, Plane<S, 2> grad, Plane<S, 8> pca,
                                                     Plane<S, 4> out, BlockMatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockMatchSmem& sm = *reinterpret_cast<BlockMatchSmem*>(smem_raw);
    constexpr bool fast = is_half<S>::value;
    const int x0 = blockIdx.x * BM_T, y0 = blockIdx.y * BM_T;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int k = tid; k < 441; k += 256) {
        const int i = k % 21 - 10, j = k / 21 - 10;
        const float d = 0.1f * sqrtf(float(i * i + j * j));
        sm.spatial[k] = expf(-2.f * d * d);
    }
    for (int k = tid; k < BM_W * BM_W; k += 256) {
        const int ty = k / BM_W, tx = k % BM_W;
        const int sx = clampi(x0 - BM_R + tx, 0, img.w - 1), sy = clampi(y0 - BM_R + ty, 0, img.h - 1);
        const f4 p = ld4<S>(img.px(sx, sy));
        sm.ycc[k] = make_float4(p.x, p.y, p.z, 0.f);
        const S* q = pca.px(sx, sy);
        if constexpr (fast) {
            const uint4 u = *reinterpret_cast<const uint4*>(q);
            const float2 a0 = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
            const float2 a1 = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
            const float2 a2 = __half22float2(*reinterpret_cast<const __half2*>(&u.z));
            const float2 a3 = __half22float2(*reinterpret_cast<const __half2*>(&u.w));
            sm.pca[k][0] = make_float4(a0.x, a0.y, a1.x, a1.y);
            sm.pca[k][1] = make_float4(a2.x, a2.y, a3.x, a3.y);
        } else {
            const float4* q4 = reinterpret_cast<const float4*>(q);
            sm.pca[k][0] = q4[0];
            sm.pca[k][1] = q4[1];
        }
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= img.w || y >= img.h) return;
    const int c0 = (threadIdx.y + BM_R) * BM_W + threadIdx.x + BM_R;
    const float4 in = sm.ycc[c0];
    const float4 ip0 = sm.pca[c0][0], ip1 = sm.pca[c0][1];
    float ls = 1.f;
    if (a.lsc > 0.f) {
        const float cx = float(img.w / 2), cy = float(img.h / 2);
        const float dx = float(x) - cx, dy = float(y) - cy;
        const float r = sqrtf(dx * dx + dy * dy) / sqrtf(cx * cx + cy * cy);
        ls = 1.f + a.lsc * r * r;
    }
    const float sig0 = sqrtf(a.var_a[0] + a.var_b[0] * ls * in.x);
    const float sig1 = sqrtf(a.var_a[1] + a.var_b[1] * ls * in.x);
    const float sig2 = sqrtf(a.var_a[2] + a.var_b[2] * ls * in.x);
    const float dm0 = 1.f / (a.tm[0] * sig0), dm1 = 1.f / (a.tm[1] * sig1), dm2 = 1.f / (a.tm[2] * sig2);
    const f2 g = ld2<S>(grad.px(x, y));
    const float mag = sqrtf(g.x * g.x + g.y * g.y);
    const float edge = smoothstepf(2.f, 16.f, a.gradient_threshold * mag / sig0);
    const float ls_ = dm0 / (1.f + a.gradient_boost * edge);
    // luma weight exp(-2 (|dp| ls_)^2) = exp(kl |dp|^2); chroma weight
    // exp(-2 (lw^2 + (dcb*c1)^2 + (dcr*c2)^2))
    const float kl = -2.f * ls_ * ls_;
    const float c1 = dm1 / a.chroma_boost, c2 = dm2 / a.chroma_boost;
    float fy = 0.f, fcb = 0.f, fcr = 0.f, ny = 0.f, nc = 0.f;
    for (int j = 0; j < 21; j++) {
        const int rowb = (threadIdx.y + j) * BM_W + threadIdx.x;
#pragma unroll 3
        for (int i = 0; i < 21; i++) {
            const int k = rowb + i;
            const float4 p0 = sm.pca[k][0], p1 = sm.pca[k][1];
            const float4 s = sm.ycc[k];
            float d, d2;
            d = p0.x - ip0.x; d2 = d * d;
            d = p0.y - ip0.y; d2 += d * d;
            d = p0.z - ip0.z; d2 += d * d;
            d = p0.w - ip0.w; d2 += d * d;
            d = p1.x - ip1.x; d2 += d * d;
            d = p1.y - ip1.y; d2 += d * d;
            d = p1.z - ip1.z; d2 += d * d;
            d = p1.w - ip1.w; d2 += d * d;
            const float lw = fast ? __expf(kl * d2) : expf(kl * d2);
            const float e1 = (s.y - in.y) * c1, e2 = (s.z - in.z) * c2;
            const float cq = lw * lw + e1 * e1 + e2 * e2;
            const float cw = fast ? __expf(-2.f * cq) : expf(-2.f * cq);
            const float sw = sm.spatial[j * 21 + i];
            const float wy = sw * lw, wc = sw * cw;
            fy += wy * s.x;
            fcb += wc * s.y;
            fcr += wc * s.z;
            ny += wy;
            nc += wc;
        }
    }
    st4<S>(out.px(x, y), f4{fy / ny, fcb / nc, fcr / nc, ny});
}

// --------------------------------------------------------------------------
// FP16-storage block matching. The reference evaluates this kernel in half
// precision (demosaic.metal:806-884); here the per-tap arithmetic is packed
// half2 and the five sums stay FP32, as in the reference:
//   * each thread owns two vertically adjacent pixels, which share 20 of
//     their 21 window rows, so every staged neighbour feeds two taps;
//   * the 8-D PCA distance runs on half2 pairs of components;
//   * both Gaussians of a neighbour for the two pixels are one packed
//     h2exp2 each (luma: exp(-2 (|dp| s)^2), chroma: exp(-2 (lw^2 + dc^2))),
//     with the constants pre-scaled by log2(e);
//   * the spatial Gaussian of the two pixels is a half2 table lookup
//     (zero where a row is outside a pixel's window).
// Tile: 32 x 16 output pixels per 256-thread block; shared memory holds
// the 52 x 36 window region as 8 PCA halves (16 B) + Y, Cb, Cr halves (8 B).
constexpr int BH_TX = 32, BH_TY = 8, BH_W = BH_TX + 20, BH_H = 2 * BH_TY + 20;

struct BlockMatchH2Smem {
    uint4 pca[BH_H * BH_W];
    uint2 ycc[BH_H * BH_W];
    __half2 sp[22 * 21];  // (weight for the upper pixel, weight for the lower pixel) per (row r, column i)
};

__device__ __forceinline__ __half2 u2h(uint32_t u) { return *reinterpret_cast<__half2*>(&u); }

template <bool UP, bool LO>
__device__ __forceinline__ void bm_row(const BlockMatchH2Smem& sm, int base, int r, const __half2 (&ip0)[4],
                                       const __half2 (&ip1)[4], float2 kl, __half2 incb, __half2 incr,
                                       __half2 c1, __half2 c2, __half2 lwk, float (&acc)[10]) {
    const __half2* sp = sm.sp + r * 21;
#pragma unroll
    for (int i = 0; i < 21; i++) {
        const uint4 P = sm.pca[base + i];
        const uint2 Y = sm.ycc[base + i];
        const __half2 p01 = u2h(P.x), p23 = u2h(P.y), p45 = u2h(P.z), p67 = u2h(P.w);
        __half d2u = __float2half(0.f), d2l = __float2half(0.f);
        if (UP) {
            __half2 a = __hsub2(p01, ip0[0]), b = __hsub2(p23, ip0[1]);
            __half2 s = __hmul2(a, a);
            s = __hfma2(b, b, s);
            a = __hsub2(p45, ip0[2]);
            b = __hsub2(p67, ip0[3]);
            s = __hfma2(a, a, s);
            s = __hfma2(b, b, s);
            d2u = __hadd(__low2half(s), __high2half(s));
        }
        if (LO) {
            __half2 a = __hsub2(p01, ip1[0]), b = __hsub2(p23, ip1[1]);
            __half2 s = __hmul2(a, a);
            s = __hfma2(b, b, s);
            a = __hsub2(p45, ip1[2]);
            b = __hsub2(p67, ip1[3]);
            s = __hfma2(a, a, s);
            s = __hfma2(b, b, s);
            d2l = __hadd(__low2half(s), __high2half(s));
        }
        // luma weights of both pixels: exp2(kl * d2). The exponent is formed in
        // FP32 (kl can exceed the half range for dark pixels; a product past
        // -65504 becomes -inf in half and exp2 gives 0, as it should).
        const __half2 lw = h2exp2(__floats2half2_rn(kl.x * __half2float(d2u), kl.y * __half2float(d2l)));
        // chroma weights: exp2(-(lw'^2 + e1'^2 + e2'^2)), primes pre-scaled by sqrt(2 log2 e)
        const __half2 ycb = u2h(Y.x), crx = u2h(Y.y);
        const __half2 e1 = __hmul2(__hsub2(__high2half2(ycb), incb), c1);
        const __half2 e2 = __hmul2(__hsub2(__low2half2(crx), incr), c2);
        const __half2 lq = __hmul2(lw, lwk);
        __half2 q = __hmul2(e2, e2);
        q = __hfma2(e1, e1, q);
        q = __hfma2(lq, lq, q);
        const __half2 cw = h2exp2(__hneg2(q));
        const __half2 s2 = sp[i];
        const float2 wy = __half22float2(__hmul2(s2, lw));
        const float2 wc = __half22float2(__hmul2(s2, cw));
        const float2 yc = __half22float2(ycb);
        const float cr = __low2float(crx);
        if (UP) {
            acc[0] = fmaf(wy.x, yc.x, acc[0]);
            acc[1] = fmaf(wc.x, yc.y, acc[1]);
            acc[2] = fmaf(wc.x, cr, acc[2]);
            acc[3] += wy.x;
            acc[4] += wc.x;
        }
        if (LO) {
            acc[5] = fmaf(wy.y, yc.x, acc[5]);
            acc[6] = fmaf(wc.y, yc.y, acc[6]);
            acc[7] = fmaf(wc.y, cr, acc[7]);
            acc[8] += wy.y;
            acc[9] += wc.y;
        }
    }
}

__global__ void __launch_bounds__(256) k_block_match_h2(Plane<__half, 4> img, Plane<__half, 2> grad,
                                                        Plane<__half, 8> pca, Plane<__half, 4> out,
                                                        BlockMatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BlockMatchH2Smem& sm = *reinterpret_cast<BlockMatchH2Smem*>(smem_raw);
    const int x0 = blockIdx.x * BH_TX, y0 = blockIdx.y * (2 * BH_TY);
    const int tid = threadIdx.y * BH_TX + threadIdx.x;
    for (int k = tid; k < 22 * 21; k += 256) {
        const int r = k / 21, i = k % 21 - 10;
        auto sw = [&](int j) {
            const float d = 0.1f * sqrtf(float(i * i + j * j));
            return expf(-2.f * d * d);
        };
        const float up = r <= 20 ? sw(r - 10) : 0.f;  // row r of the upper pixel's window is offset r - 10
        const float lo = r >= 1 ? sw(r - 11) : 0.f;   // the lower pixel's offset is r - 11
        sm.sp[k] = __floats2half2_rn(up, lo);
    }
    for (int k = tid; k < BH_W * BH_H; k += 256) {
        const int ty = k / BH_W, tx = k % BH_W;
        const int sx = clampi(x0 - 10 + tx, 0, img.w - 1), sy = clampi(y0 - 10 + ty, 0, img.h - 1);
        sm.pca[k] = *reinterpret_cast<const uint4*>(pca.px(sx, sy));
        uint2 y = *reinterpret_cast<const uint2*>(img.px(sx, sy));
        y.y &= 0xffffu;  // keep Cr, zero the w half
        sm.ycc[k] = y;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, yu = y0 + 2 * threadIdx.y;
    const float kLog2e = 1.4426950408889634f;
    __half2 ip0[4], ip1[4];
    float kl[2], c1v[2], c2v[2], incb[2], incr[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        const int c = (2 * threadIdx.y + p + 10) * BH_W + threadIdx.x + 10;
        const uint4 P = sm.pca[c];
        __half2* ip = p ? ip1 : ip0;
        ip[0] = u2h(P.x); ip[1] = u2h(P.y); ip[2] = u2h(P.z); ip[3] = u2h(P.w);
        const uint2 Y = sm.ycc[c];
        const float2 yc = __half22float2(u2h(Y.x));
        const float cr = __low2float(u2h(Y.y));
        const int py = min(yu + p, img.h - 1), px = min(x, img.w - 1);
        float ls = 1.f;
        if (a.lsc > 0.f) {
            const float cx = float(img.w / 2), cy = float(img.h / 2);
            const float dx = float(px) - cx, dy = float(py) - cy;
            const float rr = sqrtf(dx * dx + dy * dy) / sqrtf(cx * cx + cy * cy);
            ls = 1.f + a.lsc * rr * rr;
        }
        const float sig0 = sqrtf(a.var_a[0] + a.var_b[0] * ls * yc.x);
        const float sig1 = sqrtf(a.var_a[1] + a.var_b[1] * ls * yc.x);
        const float sig2 = sqrtf(a.var_a[2] + a.var_b[2] * ls * yc.x);
        const float dm0 = 1.f / (a.tm[0] * sig0), dm1 = 1.f / (a.tm[1] * sig1), dm2 = 1.f / (a.tm[2] * sig2);
        const f2 g = ld2<__half>(grad.px(px, py));
        const float mag = sqrtf(g.x * g.x + g.y * g.y);
        const float edge = smoothstepf(2.f, 16.f, a.gradient_threshold * mag / sig0);
        const float lsc_ = dm0 / (1.f + a.gradient_boost * edge);
        kl[p] = -2.f * kLog2e * lsc_ * lsc_;
        const float sq = sqrtf(2.f * kLog2e);
        c1v[p] = sq * dm1 / a.chroma_boost;
        c2v[p] = sq * dm2 / a.chroma_boost;
        incb[p] = yc.y;
        incr[p] = cr;
    }
    const float2 klh = make_float2(fmaxf(kl[0], -1e30f), fmaxf(kl[1], -1e30f));
    // chroma scales saturate at the half maximum (a difference of one half
    // ulp times 65504 already zeroes the weight)
    const __half2 c1h = __floats2half2_rn(fminf(c1v[0], 65504.f), fminf(c1v[1], 65504.f));
    const __half2 c2h = __floats2half2_rn(fminf(c2v[0], 65504.f), fminf(c2v[1], 65504.f));
    const __half2 incbh = __floats2half2_rn(incb[0], incb[1]), incrh = __floats2half2_rn(incr[0], incr[1]);
    const __half2 lwk = __float2half2_rn(sqrtf(2.f * kLog2e));
    float acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    // window rows of the pair: r = 0 (upper only), 1..20 (both), 21 (lower only)
    const int col = threadIdx.x;
    const int row0 = 2 * threadIdx.y;
    bm_row<true, false>(sm, (row0 + 0) * BH_W + col, 0, ip0, ip1, klh, incbh, incrh, c1h, c2h, lwk, acc);
    for (int r = 1; r <= 20; r++)
        bm_row<true, true>(sm, (row0 + r) * BH_W + col, r, ip0, ip1, klh, incbh, incrh, c1h, c2h, lwk, acc);
    bm_row<false, true>(sm, (row0 + 21) * BH_W + col, 21, ip0, ip1, klh, incbh, incrh, c1h, c2h, lwk, acc);
    if (x < out.w) {
        if (yu < out.h) st4<__half>(out.px(x, yu), f4{acc[0] / acc[3], acc[1] / acc[4], acc[2] / acc[4], acc[3]});
        if (yu + 1 < out.h)
            st4<__half>(out.px(x, yu + 1), f4{acc[5] / acc[8], acc[6] / acc[9], acc[7] / acc[9], acc[8]});
    }
}

// ------------------------------------------------------------------ launchers
static inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

template <class S, int C>
void launch_downsample(Plane<S, C> in, Plane<S, C> out, cudaStream_t s) {
    dim3 b(32, 8);
    k_downsample<S, C><<<grid2(out.w, out.h, b), b, 0, s>>>(in, out, float(in.w) / float(out.w),
                                                            float(in.h) / float(out.h));
}

template <class S>
void launch_subtract_noise(Plane<S, 4> in, Plane<S, 4> coarse, Plane<S, 4> coarse_den, Plane<S, 2> grad,
                           Plane<S, 4> out, const SubtractArgs& a, cudaStream_t s) {
    dim3 b(32, 8);
    k_subtract_noise<S><<<grid2(in.w, in.h, b), b, 0, s>>>(in, coarse, coarse_den, grad, out, a,
                                                          float(coarse.w) / float(in.w), float(coarse.h) / float(in.h));
}

static void init_pairs() {
    static bool done = false;
    if (done) return;
    uint8_t r[325], c[325];
    int k = 0;
    for (int i = 0; i < 25; i++)
        for (int j = i; j < 25; j++, k++) {
            r[k] = uint8_t(i);
            c[k] = uint8_t(j);
        }
    cudaMemcpyToSymbol(kPairR, r, sizeof(r));
    cudaMemcpyToSymbol(kPairC, c, sizeof(c));
    done = true;
}

int pca_cov_blocks(int w, int h) {
    const int n = (w / 8) * (h / 8);
    return n <= 0 ? 0 : std::max(1, std::min(kPcaMaxBlocks, (n + PC_CHUNK - 1) / PC_CHUNK));
}

template <class S>
void launch_pca_cov(Plane<S, 4> img, double* part, cudaStream_t s) {
    init_pairs();
    const int blocks = pca_cov_blocks(img.w, img.h);
    if (blocks == 0) return;
    k_pca_cov<S><<<blocks, 352, 0, s>>>(img, part);
}

void launch_pca_eigen(const double* part, int n_blocks, int n_patches, float* basis, int* status, cudaStream_t s) {
    k_pca_eigen<<<1, 1024, 0, s>>>(part, n_blocks, n_patches, basis, status);
}

template <class S>
void launch_pca_project(Plane<S, 4> img, const float* basis, Plane<S, 8> out, cudaStream_t s) {
    dim3 b(32, 8);
    k_pca_project<S><<<grid2(img.w, img.h, b), b, 0, s>>>(img, basis, out);
}

template <class S>
void launch_block_match(Plane<S, 4> img, Plane<S, 2> grad, Plane<S, 8> pca, Plane<S, 4> out, const BlockMatchArgs& a,
                        cudaStream_t s) {
    if constexpr (is_half<S>::value) {
        static bool attr_h = false;
        if (!attr_h) {
            cudaFuncSetAttribute(k_block_match_h2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(BlockMatchH2Smem)));
            attr_h = true;
        }
        dim3 b(BH_TX, BH_TY);
        dim3 g((img.w + BH_TX - 1) / BH_TX, (img.h + 2 * BH_TY - 1) / (2 * BH_TY));
        k_block_match_h2<<<g, b, sizeof(BlockMatchH2Smem), s>>>(img, grad, pca, out, a);
    } else {
        static bool attr = false;
        if (!attr) {
            cudaFuncSetAttribute(k_block_match<S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(BlockMatchSmem)));
            attr = true;
        }
        dim3 b(BM_T, BM_T);
        k_block_match<S><<<grid2(img.w, img.h, b), b, sizeof(BlockMatchSmem), s>>>(img, grad, pca, out, a);
    }
}

// Host FP64 eigen-solve of the same accumulators: the per-level host PCA of
// the reference (pyramid_processor.cpp:148-149), for the GLS_HOST_PCA path.
void host_pca_basis(const double* part, int n_blocks, int n_patches, float* basis) {
    double acc[kPcaAcc];
    for (int t = 0; t < kPcaAcc; t++) {
        double v = 0.0;
        for (int b = 0; b < n_blocks; b++) v += part[b * kPcaAcc + t];
        acc[t] = v;
    }
    if (n_patches < 2) {
        for (int t = 0; t < 200; t++) basis[t] = ((t / 8) == (t % 8)) ? 1.f : 0.f;
        return;
    }
    double A[25][25], V[25][25];
    const double n = double(n_patches);
    for (int i = 0; i < 25; i++)
        for (int j = 0; j < 25; j++) {
            const int r = std::min(i, j), c = std::max(i, j);
            const int idx = r * 25 - r * (r - 1) / 2 + (c - r);
            A[i][j] = (acc[idx] - n * (acc[325 + i] / n) * (acc[325 + j] / n)) / (n - 1.0);
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < 25; i++)
            for (int j = 0; j < 25; j++) {
                tot += A[i][j] * A[i][j];
                if (i != j) off += A[i][j] * A[i][j];
            }
        if (off <= 1e-26 * tot || off == 0) break;
        for (int p = 0; p < 24; p++)
            for (int q = p + 1; q < 25; q++) {
                const double apq = A[p][q];
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (A[q][q] - A[p][p]) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < 25; k++) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 25; k++) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 25; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    int order[25];
    for (int k = 0; k < 25; k++) order[k] = k;
    for (int k = 1; k < 25; k++) {
        const int e = order[k];
        int m = k - 1;
        while (m >= 0 && A[order[m]][order[m]] < A[e][e]) {
            order[m + 1] = order[m];
            m--;
        }
        order[m + 1] = e;
    }
    double ev[25], evec[25 * 25], work[200];
    for (int c = 0; c < 25; c++) {
        ev[c] = A[order[c]][order[c]];
        for (int r = 0; r < 25; r++) evec[r * 25 + c] = V[r][order[c]];
    }
    select_pca_basis(ev, evec, 25, work, basis);
}

#define GLS_INST(S)                                                                                              \
    template void launch_downsample<S, 4>(Plane<S, 4>, Plane<S, 4>, cudaStream_t);                              \
    template void launch_downsample<S, 2>(Plane<S, 2>, Plane<S, 2>, cudaStream_t);                              \
    template void launch_subtract_noise<S>(Plane<S, 4>, Plane<S, 4>, Plane<S, 4>, Plane<S, 2>, Plane<S, 4>,     \
                                           const SubtractArgs&, cudaStream_t);                                   \
    template void launch_pca_cov<S>(Plane<S, 4>, double*, cudaStream_t);                                         \
    template void launch_pca_project<S>(Plane<S, 4>, const float*, Plane<S, 8>, cudaStream_t);                  \
    template void launch_block_match<S>(Plane<S, 4>, Plane<S, 2>, Plane<S, 8>, Plane<S, 4>,                     \
                                        const BlockMatchArgs&, cudaStream_t);
GLS_INST(float)
GLS_INST(__half)
#undef GLS_INST

}  // namespace gls
