// gls_pyramid.cu — kernels of PyramidProcessor<levels>::denoise
// (pyramid_processor.cpp:96-172): Gaussian-pyramid downsample, the
// reconstruct (noise subtraction) step, the per-level PCA patch basis
// (covariance + FP64 tridiagonal eigen-solve on the device; two-sided
// Jacobi on the host for GLS_HOST_PCA) and the 5x5-patch
// PCA projection. The block-matching denoise is in gls_blockmatch.cu.
#include <cmath>
#include <cstdio>

#include "gls_common.cuh"
#include "gls_kernels.h"
#include "gls_pca_pairs.h"
#include "gls_pyramid_dev.cuh"

namespace gls {

// --------------------------------------------------------------------------
// downsampleImageXYZ / downsampleImageXY, demosaic.metal:886-920: mean of
// four bilinear samples at texel-space (x*r - 0.5, (x+1)*r - 0.5) with
// r = in/out size (a 4x4 box for an exact halving). Positions are formed
// with explicit FP32 roundings, matching the oracle's FP32 run.
template <class S, int C>
__device__ __forceinline__ void downsample_px(const Plane<S, C>& in, const Plane<S, C>& out, float rx, float ry,
                                              int x, int y) {
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

template <class S, int C>
__global__ void __launch_bounds__(256) k_downsample(Plane<S, C> in, Plane<S, C> out, float rx, float ry) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= out.w || y >= out.h) return;
    downsample_px<S, C>(in, out, rx, ry, x, y);
}

// The image and the gradient of a pyramid level in one launch (same sizes,
// same sample positions): PyramidProcessor::denoise's two downsamples
// (pyramid_processor.cpp:109-110).
template <class S>
__global__ void __launch_bounds__(256) k_downsample_pair(Plane<S, 4> img, Plane<S, 4> img_out, Plane<S, 2> grad,
                                                         Plane<S, 2> grad_out, float rx, float ry) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= img_out.w || y >= img_out.h) return;
    downsample_px<S, 4>(img, img_out, rx, ry, x, y);
    downsample_px<S, 2>(grad, grad_out, rx, ry, x, y);
}

template <class S>
__global__ void __launch_bounds__(256) k_subtract_noise(Plane<S, 4> in, Plane<S, 4> coarse, Plane<S, 4> coarse_den,
                                                        Plane<S, 2> grad, Plane<S, 4> out, SubtractArgs a, float rx,
                                                        float ry) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= in.w || y >= in.h) return;
    subtract_noise_px<S>(in, coarse, coarse_den, grad, out, a, rx, ry, x, y);
}

template <class S>
__global__ void __launch_bounds__(352, 3) k_pca_cov(Plane<S, 4> img, double* __restrict__ part, int group, int n_chunks) {
    __shared__ CovSmem sm;
    const int c0 = blockIdx.x * group;
    pca_cov_row<S>(img, part + size_t(blockIdx.x) * kPcaAcc, c0, min(c0 + group, n_chunks), sm);
}

constexpr int EJ_THREADS = 704;  // 22 warps: the prologue's 700 partial sums at once

__global__ void __launch_bounds__(EJ_THREADS) k_pca_eigen(const double* __restrict__ part, int n_blocks,
                                                         int n_patches, float* __restrict__ basis, int* status) {
    __shared__ EigenSmem sm;
    pca_eigen_block(part, n_blocks, n_patches, basis, status, sm);
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
void launch_downsample_pair(Plane<S, 4> img, Plane<S, 4> img_out, Plane<S, 2> grad, Plane<S, 2> grad_out,
                            cudaStream_t s) {
    dim3 b(32, 8);
    k_downsample_pair<S><<<grid2(img_out.w, img_out.h, b), b, 0, s>>>(
        img, img_out, grad, grad_out, float(img.w) / float(img_out.w), float(img.h) / float(img_out.h));
}

template <class S>
void launch_subtract_noise(Plane<S, 4> in, Plane<S, 4> coarse, Plane<S, 4> coarse_den, Plane<S, 2> grad,
                           Plane<S, 4> out, const SubtractArgs& a, cudaStream_t s) {
    dim3 b(32, 8);
    k_subtract_noise<S><<<grid2(in.w, in.h, b), b, 0, s>>>(in, coarse, coarse_den, grad, out, a,
                                                          float(coarse.w) / float(in.w), float(coarse.h) / float(in.h));
}

int pca_cov_chunks(int w, int h) {
    const int n = (w / 8) * (h / 8);
    return n <= 0 ? 0 : (n + PC_CHUNK - 1) / PC_CHUNK;
}

int pca_cov_rows(int w, int h) {
    const int chunks = pca_cov_chunks(w, h), g = pca_cov_group(chunks);
    return (chunks + g - 1) / g;
}

template <class S>
void launch_pca_cov(Plane<S, 4> img, double* part, cudaStream_t s) {
    const int rows = pca_cov_rows(img.w, img.h);
    if (rows == 0) return;
    const int chunks = pca_cov_chunks(img.w, img.h);
    k_pca_cov<S><<<rows, 352, 0, s>>>(img, part, pca_cov_group(chunks), chunks);
}

template <class S>
void launch_pca_cov_rows(Plane<S, 4> img, double* part, int rows, cudaStream_t s) {
    if (rows > 0) k_pca_cov<S><<<rows, 352, 0, s>>>(img, part, 1, pca_cov_chunks(img.w, img.h));
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
    template void launch_downsample_pair<S>(Plane<S, 4>, Plane<S, 4>, Plane<S, 2>, Plane<S, 2>, cudaStream_t);  \
    template void launch_subtract_noise<S>(Plane<S, 4>, Plane<S, 4>, Plane<S, 4>, Plane<S, 2>, Plane<S, 4>,     \
                                           const SubtractArgs&, cudaStream_t);                                   \
    template void launch_pca_cov<S>(Plane<S, 4>, double*, cudaStream_t);                                         \
    template void launch_pca_project<S>(Plane<S, 4>, const float*, Plane<S, 8>, cudaStream_t);
GLS_INST(float)
GLS_INST(__half)
#undef GLS_INST

}  // namespace gls
