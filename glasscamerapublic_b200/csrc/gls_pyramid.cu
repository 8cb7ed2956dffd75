// gls_pyramid.cu — kernels of PyramidProcessor<levels>::denoise
// (pyramid_processor.cpp:96-172): Gaussian-pyramid downsample, the
// reconstruct (noise subtraction) step, the per-level PCA patch basis
// (covariance + FP64 Jacobi eigen-solve on the device) and the 5x5-patch
// PCA projection. The block-matching denoise is in gls_blockmatch.cu.
#include <cmath>
#include <cstdio>

#include "gls_common.cuh"
#include "gls_kernels.h"
#include "gls_pca_pairs.h"

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
// scheduling (no atomics). A thread finds its (r, c) from its index
// (pca_pair), so the kernel needs no table loaded per device.

constexpr int PC_CHUNK = 64;

template <class S>
__global__ void __launch_bounds__(352) k_pca_cov(Plane<S, 4> img, double* __restrict__ part) {
    __shared__ float sp[PC_CHUNK][kPcaDim + 1];
    const int gw = img.w / 8, gh = img.h / 8;
    const int n = gw * gh;
    const int t = threadIdx.x;
    double sum = 0.0;
    int r = 0, c = 0;
    if (t < kPcaTri) {
        pca_pair(t, r, c);
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
// SelfAdjointEigenSolver, PCA.cpp:36): one-sided (Hestenes) Jacobi in FP64,
// one warp. Lane j holds column j of the covariance in registers; a
// round-robin schedule (25 columns + one empty, 13 disjoint pairs per
// round, 25 rounds per sweep) pairs the lanes, the partner's column comes
// by shuffles, and both lanes of a pair form the same rotation from the
// two columns' Gram entries (alpha, beta, gamma) and rotate their own
// column. A sweep without a rotation (|gamma| <= 1e-14 sqrt(alpha beta)
// for every pair) ends the solve; at most 40 sweeps, so the kernel always
// ends. The covariance C is symmetric positive semi-definite, so the
// converged columns are C V = Q Lambda: eigenvalue j is the norm of
// column j and its eigenvector the normalised column. The top-8
// eigenvectors (descending eigenvalue, each signed so its largest-magnitude
// entry is positive) are written as a row-major 25x8 FP32 basis. status
// receives the sweep count, or -1 when the sweep limit was hit.
constexpr int EJ_THREADS = 352;

__device__ __forceinline__ void jacobi_rotation(double app, double aqq, double apq, double& c, double& s) {
    // The angle needs only FP32 accuracy: a rotation a little off the exact
    // one leaves gamma at about 1e-7 of its value, which later sweeps
    // remove. It has to be orthogonal to FP64 precision, which two Newton
    // steps for 1 / sqrt(c^2 + s^2) from 1 restore.
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(2.0 * apq));
    const float th = float((aqq - app) * r);
    const float at = fabsf(th);
    float tt = at < 1e18f ? __fdividef(1.f, at + sqrtf(fmaf(at, at, 1.f))) : 0.5f / at;
    tt = copysignf(tt, th);
    const float c32 = rsqrtf(fmaf(tt, tt, 1.f));
    const double cd = c32, sd = double(tt * c32);
    const double n2 = cd * cd + sd * sd;
    double y = 1.5 - 0.5 * n2;
    y = y * (1.5 - 0.5 * n2 * y * y);
    c = cd * y;
    s = sd * y;
}

__global__ void __launch_bounds__(EJ_THREADS) k_pca_eigen(const double* __restrict__ part, int n_blocks,
                                                         int n_patches, float* __restrict__ basis, int* status) {
    __shared__ double acc[kPcaAcc];
    __shared__ double C[25][25];          // covariance
    __shared__ double U[25][26];          // normalised final columns (column j = lane j)
    __shared__ double B[25][26];          // eigenvectors, column c = the c-th largest
    __shared__ double ev_l[25], ev[25], work[200];
    __shared__ int order[25];
    const int t = threadIdx.x;

    if (n_patches < 2) {
        for (int k = t; k < 25 * 8; k += blockDim.x) basis[k] = ((k / 8) == (k % 8)) ? 1.f : 0.f;
        if (t == 0 && status) *status = 0;
        return;
    }
    // block partials summed in block order (deterministic), eight loads in flight
    if (t < kPcaAcc) {
        double v = 0.0;
        int b = 0;
        for (; b + 8 <= n_blocks; b += 8) {
            double x[8];
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = part[(b + k) * kPcaAcc + t];
#pragma unroll
            for (int k = 0; k < 8; k++) v += x[k];
        }
        for (; b < n_blocks; b++) v += part[b * kPcaAcc + t];
        acc[t] = v;
    }
    __syncthreads();
    // covariance from raw moments
    for (int k = t; k < 625; k += blockDim.x) {
        const int i = k / 25, j = k % 25;
        const int r = min(i, j), c = max(i, j);
        const int idx = pca_tri_index(r, c);
        const double n = double(n_patches);
        const double mi = acc[325 + i] / n, mj = acc[325 + j] / n;
        C[i][j] = (acc[idx] - n * mi * mj) / (n - 1.0);
    }
    __syncthreads();
    if (t >= 32) return;  // one warp solves
    const int lane = t;
    double a[25];
#pragma unroll
    for (int r = 0; r < 25; r++) a[r] = lane < 25 ? C[r][lane] : 0.0;
    int sweep = 0;
    for (; sweep < 40; sweep++) {
        bool rotated = false;
#pragma unroll 1
        for (int round = 0; round < 25; round++) {
            // pairs of this round: (round, 25) and the lanes whose indices sum to 2 round (mod 25)
            int partner = lane;
            if (lane < 25) partner = lane == round ? 25 : (2 * round - lane + 50) % 25;
            else if (lane == 25) partner = round;
            double b[25];
#pragma unroll
            for (int r = 0; r < 25; r++) b[r] = __shfl_sync(0xffffffffu, a[r], partner);
            // Gram entries, two partial sums each (the same order in both lanes of a pair)
            double al0 = 0, al1 = 0, be0 = 0, be1 = 0, ga0 = 0, ga1 = 0;
#pragma unroll
            for (int r = 0; r < 24; r += 2) {
                al0 = fma(a[r], a[r], al0);
                be0 = fma(b[r], b[r], be0);
                ga0 = fma(a[r], b[r], ga0);
                al1 = fma(a[r + 1], a[r + 1], al1);
                be1 = fma(b[r + 1], b[r + 1], be1);
                ga1 = fma(a[r + 1], b[r + 1], ga1);
            }
            const double al = fma(a[24], a[24], al0 + al1), be = fma(b[24], b[24], be0 + be1);
            const double ga = fma(a[24], b[24], ga0 + ga1);
            const bool low = lane < partner;
            if (partner < 25 && lane < 25 && partner != lane && ga * ga > 1e-28 * al * be && fabs(ga) >= 1e-300) {
                double c, s;
                jacobi_rotation(low ? al : be, low ? be : al, ga, c, s);
                rotated = true;
                // the lower index p: c a_p - s a_q; the higher q: s a_p + c a_q
#pragma unroll
                for (int r = 0; r < 25; r++) a[r] = low ? fma(c, a[r], -s * b[r]) : fma(s, b[r], c * a[r]);
            }
        }
        if (!__any_sync(0xffffffffu, rotated)) break;
    }
    if (lane < 25) {
        double nn = 0.0;
#pragma unroll
        for (int r = 0; r < 25; r++) nn = fma(a[r], a[r], nn);
        const double e = sqrt(nn);
        const double inv = e > 0.0 ? 1.0 / e : 0.0;
        ev_l[lane] = e;
#pragma unroll
        for (int r = 0; r < 25; r++) U[r][lane] = a[r] * inv;
    }
    __syncwarp();
    // order eigenvalues descending (stable by index)
    if (lane == 0) {
        for (int k = 0; k < 25; k++) order[k] = k;
        for (int k = 1; k < 25; k++) {  // insertion sort, stable
            const int e = order[k];
            int m = k - 1;
            while (m >= 0 && ev_l[order[m]] < ev_l[e]) {
                order[m + 1] = order[m];
                m--;
            }
            order[m + 1] = e;
        }
        if (status) *status = sweep < 40 ? sweep : -1;
    }
    __syncwarp();
    if (lane < 25) ev[lane] = ev_l[order[lane]];
    for (int k = lane; k < 625; k += 32) B[k / 25][k % 25] = U[k / 25][order[k % 25]];
    __syncwarp();
    if (lane == 0) select_pca_basis(ev, &B[0][0], 26, work, basis);
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

int pca_cov_blocks(int w, int h) {
    const int n = (w / 8) * (h / 8);
    return n <= 0 ? 0 : std::max(1, std::min(kPcaMaxBlocks, (n + PC_CHUNK - 1) / PC_CHUNK));
}

template <class S>
void launch_pca_cov(Plane<S, 4> img, double* part, cudaStream_t s) {
    const int blocks = pca_cov_blocks(img.w, img.h);
    if (blocks == 0) return;
    k_pca_cov<S><<<blocks, 352, 0, s>>>(img, part);
}

template <class S>
void launch_pca_cov_rows(Plane<S, 4> img, double* part, int rows, cudaStream_t s) {
    if (rows > 0) k_pca_cov<S><<<rows, 352, 0, s>>>(img, part);
}
template void launch_pca_cov_rows<float>(Plane<float, 4>, double*, int, cudaStream_t);
template void launch_pca_cov_rows<__half>(Plane<__half, 4>, double*, int, cudaStream_t);

void launch_pca_eigen(const double* part, int n_blocks, int n_patches, float* basis, int* status, cudaStream_t s) {
    k_pca_eigen<<<1, EJ_THREADS, 0, s>>>(part, n_blocks, n_patches, basis, status);
}

template <class S>
void launch_pca_project(Plane<S, 4> img, const float* basis, Plane<S, 8> out, cudaStream_t s) {
    dim3 b(32, 8);
    k_pca_project<S><<<grid2(img.w, img.h, b), b, 0, s>>>(img, basis, out);
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
            const int idx = pca_tri_index(r, c);
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
    template void launch_pca_project<S>(Plane<S, 4>, const float*, Plane<S, 8>, cudaStream_t);
GLS_INST(float)
GLS_INST(__half)
#undef GLS_INST

}  // namespace gls
