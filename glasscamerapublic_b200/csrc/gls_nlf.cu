// gls_nlf.cu — noise-model measurement of RawConverter with
// calibrateFromImage:
//   * k_raw_stats    basicRawNoiseStatistics (demosaic.metal:1110-1136): the
//                    9x9 mean and variance of the four raw channels at every
//                    half-resolution position, from a shared-memory tile
//   * k_ycc_stats    basicNoiseStatistics (:1138-1159): the 5x5 mean of Y
//                    and variances of Y, Cb, Cr at every position of a level
//   * k_fit_pass /   the two-pass least-squares fits of MeasureRawNLF
//     k_fit_finish   (raw_converter.cpp:339-490) and MeasureYCbCrNLF
//                    (pyramid_processor.cpp:173-324) on the device: each
//                    pass sums over the statistics in FP64 (fixed grid, block
//                    partial sums in a fixed order, so the result does not
//                    depend on scheduling) and a one-block kernel forms the
//                    fit from the partial sums
// The statistics are FP32 operation for operation as in the reference
// kernels (one rounding per operation, no contraction), so the FP32 path's
// statistics equal the CPU oracle's bit for bit; the fits agree with the
// oracle's sequential FP64 sums to their last bits.
#include <cmath>

#include "../../include/glscam.h"
#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

namespace {

// ---------------------------------------------------------------- statistics
constexpr int RS_TX = 32, RS_TY = 8;                     // half-resolution positions per block
constexpr int RS_W = 2 * RS_TX + 10, RS_H = 2 * RS_TY + 10;  // full-resolution tile: 2x + [-4, 5]

template <class S>
__global__ void __launch_bounds__(RS_TX* RS_TY) k_raw_stats(Plane<S, 1> raw, int pattern, Plane<float, 4> mean,
                                                            Plane<float, 4> var) {
    __shared__ float tile[RS_H][RS_W];
    const int X0 = blockIdx.x * RS_TX, Y0 = blockIdx.y * RS_TY;  // half-resolution origin
    const int tid = threadIdx.y * RS_TX + threadIdx.x;
    for (int k = tid; k < RS_W * RS_H; k += RS_TX * RS_TY) {
        const int ty = k / RS_W, tx = k % RS_W;
        tile[ty][tx] = to_f(*raw.pxc(2 * X0 - 4 + tx, 2 * Y0 - 4 + ty));
    }
    __syncthreads();
    const int x = X0 + threadIdx.x, y = Y0 + threadIdx.y;
    if (x >= mean.w || y >= mean.h) return;
    int ox[4], oy[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        ox[c] = kBayer[pattern][c][0];
        oy[c] = kBayer[pattern][c][1];
    }
    float sum[4] = {0.f, 0.f, 0.f, 0.f}, sumSq[4] = {0.f, 0.f, 0.f, 0.f};
    // the window steps one full-resolution pixel from 2 (x, y) and reads each
    // channel at its Bayer offset from there (readRAWQuad)
    const int bx0 = 2 * threadIdx.x, by0 = 2 * threadIdx.y;  // tile position of 2 (x, y) - 4
    for (int dy = 0; dy < 9; dy++)
#pragma unroll
        for (int dx = 0; dx < 9; dx++)
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float s = tile[by0 + dy + oy[c]][bx0 + dx + ox[c]];
                sum[c] = __fadd_rn(sum[c], s);
                sumSq[c] = __fadd_rn(sumSq[c], __fmul_rn(s, s));
            }
    f4 m, v;
    float* mp = &m.x;
    float* vp = &v.x;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        mp[c] = __fdiv_rn(sum[c], 81.f);
        vp[c] = __fdiv_rn(__fsub_rn(sumSq[c], __fdiv_rn(__fmul_rn(sum[c], sum[c]), 81.f)), 81.f);
    }
    st4<float>(mean.px(x, y), m);
    st4<float>(var.px(x, y), v);
}

constexpr int YS_TX = 32, YS_TY = 8;
constexpr int YS_W = YS_TX + 4, YS_H = YS_TY + 4;

template <class S>
__global__ void __launch_bounds__(YS_TX* YS_TY) k_ycc_stats(Plane<S, 4> img, Plane<float, 4> stats) {
    __shared__ float3 tile[YS_H][YS_W];
    const int x0 = blockIdx.x * YS_TX, y0 = blockIdx.y * YS_TY;
    const int tid = threadIdx.y * YS_TX + threadIdx.x;
    for (int k = tid; k < YS_W * YS_H; k += YS_TX * YS_TY) {
        const int ty = k / YS_W, tx = k % YS_W;
        const f4 p = ld4<S>(img.pxc(x0 - 2 + tx, y0 - 2 + ty));
        tile[ty][tx] = make_float3(p.x, p.y, p.z);
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= img.w || y >= img.h) return;
    float sum[3] = {0.f, 0.f, 0.f}, sumSq[3] = {0.f, 0.f, 0.f};
    for (int dy = 0; dy < 5; dy++)
#pragma unroll
        for (int dx = 0; dx < 5; dx++) {
            const float3 t = tile[threadIdx.y + dy][threadIdx.x + dx];
            const float s[3] = {t.x, t.y, t.z};
#pragma unroll
            for (int c = 0; c < 3; c++) {
                sum[c] = __fadd_rn(sum[c], s[c]);
                sumSq[c] = __fadd_rn(sumSq[c], __fmul_rn(s[c], s[c]));
            }
        }
    f4 o;
    o.x = __fdiv_rn(sum[0], 25.f);
    float* op = &o.y;
#pragma unroll
    for (int c = 0; c < 3; c++) op[c] = __fdiv_rn(__fsub_rn(sumSq[c], __fdiv_rn(__fmul_rn(sum[c], sum[c]), 25.f)), 25.f);
    st4<float>(stats.px(x, y), o);
}

// ---------------------------------------------------------------- fits
// raw: mean and var planes, a regressor per channel (4 channels);
// ycc: one statistics plane (mean Y, var Y, Cb, Cr), the luma mean the
// regressor of all three variances
struct FitInput {
    const float4* mean;  // raw: means; ycc: the statistics
    const float4* var;   // raw: variances; ycc: unused
    int w, h;
    size_t pitch;  // float4 per row
    int raw;       // 1: MeasureRawNLF, 0: MeasureYCbCrNLF
    double pixels;  // raw: the raw frame's pixel count; ycc: the level's
    float exposure;
};

constexpr int FIT_BLOCKS = 296, FIT_THREADS = 256, FIT_K = 24;

struct Sample {
    double m[4], v[4];
};

__device__ __forceinline__ Sample load_sample(const FitInput& in, int x, int y) {
    Sample s;
    if (in.raw) {
        const float4 m = in.mean[size_t(y) * in.pitch + x], v = in.var[size_t(y) * in.pitch + x];
        s.m[0] = m.x, s.m[1] = m.y, s.m[2] = m.z, s.m[3] = m.w;
        s.v[0] = v.x, s.v[1] = v.y, s.v[2] = v.z, s.v[3] = v.w;
    } else {
        const float4 t = in.mean[size_t(y) * in.pitch + x];
        s.m[0] = s.m[1] = s.m[2] = s.m[3] = t.x;
        s.v[0] = t.y, s.v[1] = t.z, s.v[2] = t.w, s.v[3] = 0.0;
    }
    return s;
}

__device__ __forceinline__ int nch(const FitInput& in) { return in.raw ? 4 : 3; }

// a position counts in the fits: no NaN, every mean in [0.001, 0.9] and
// every variance within the bound
__device__ __forceinline__ bool usable(const FitInput& in, const Sample& s, const double* bound) {
    const int n = nch(in);
    bool ok = true;
#pragma unroll
    for (int c = 0; c < 4; c++)
        if (c < n) ok = ok && !isnan(s.m[c]) && !isnan(s.v[c]);
#pragma unroll
    for (int c = 0; c < 4; c++)
        if (c < n) ok = ok && s.m[c] >= 0.001 && s.m[c] <= 0.9 && s.v[c] <= bound[c];
    return ok;
}

// the variance class 6 + trunc(clamp(log10(largest), -6, -1)) of a
// position, or -1 where it has none (a NaN or, for the YCbCr fit, a
// non-positive variance; a NaN largest value, which the reference turns
// into an undefined histogram index)
__device__ __forceinline__ int variance_class(const FitInput& in, const Sample& s) {
    const int n = nch(in);
    bool valid = true;
#pragma unroll
    for (int c = 0; c < 4; c++)
        if (c < n) valid = valid && !isnan(s.v[c]) && (in.raw || s.v[c] > 0.0);
    if (!valid) return -1;
    double m = log10(s.v[0]);
#pragma unroll
    for (int c = 1; c < 4; c++)
        if (c < n) {
            const double l = log10(s.v[c]);
            if (l > m) m = l;
        }
    if (isnan(m)) return -1;
    return 6 + int(fmin(fmax(m, -6.0), -1.0));
}

struct FitState {
    double bound[4];
    double A[4], B[4];
    double err2[4];
    double N1;
};

__device__ __forceinline__ double max_s(double v, double s) { return v > s ? v : s; }

// pass: 0 the class histogram; 1 the first fit's sums; 2 its squared
// residuals; 3 the second fit's sums and squared residuals
template <int PASS>
__global__ void __launch_bounds__(FIT_THREADS) k_fit_pass(FitInput in, const FitState* __restrict__ st_,
                                                          double* __restrict__ partial) {
    __shared__ double red[FIT_THREADS];
    double acc[FIT_K];
#pragma unroll
    for (int k = 0; k < FIT_K; k++) acc[k] = 0.0;
    FitState st;
    if (PASS > 0) st = *st_;
    const int n = nch(in);
    const long total = long(in.w) * in.h;
    for (long i = long(blockIdx.x) * FIT_THREADS + threadIdx.x; i < total; i += long(FIT_BLOCKS) * FIT_THREADS) {
        const int x = int(i % in.w), y = int(i / in.w);
        const Sample s = load_sample(in, x, y);
        if (PASS == 0) {
            const int k = variance_class(in, s);
#pragma unroll
            for (int j = 0; j < 6; j++)
                if (k == j) acc[j] += 1.0;
        } else if (PASS == 1 || PASS == 2) {
            if (!usable(in, s, st.bound)) continue;
            if (PASS == 1) {
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (c < n) {
                        acc[c] += s.m[c];
                        acc[4 + c] += s.v[c];
                        acc[8 + c] += s.m[c] * s.m[c];
                        acc[12 + c] += s.m[c] * s.v[c];
                    }
                acc[16] += 1.0;
            } else {
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (c < n) {
                        const double d = (st.A[c] + st.B[c] * s.m[c]) - s.v[c];
                        acc[c] += d * d;
                    }
            }
        } else {
            if (!usable(in, s, st.bound)) continue;
            double d2[4];
            bool fits = true;
            const double f = in.raw ? 0.5 : 1.0;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                d2[c] = 0.0;
                if (c < n) {
                    const double d = fabs((st.A[c] + st.B[c] * s.m[c]) - s.v[c]);
                    d2[c] = d * d;
                    fits = fits && d2[c] <= f * st.err2[c];
                }
            }
            if (fits) {
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (c < n) {
                        acc[c] += s.m[c];
                        acc[4 + c] += s.v[c];
                        acc[8 + c] += s.m[c] * s.m[c];
                        acc[12 + c] += s.m[c] * s.v[c];
                        acc[17 + c] += d2[c];
                    }
                acc[16] += 1.0;
            }
        }
    }
    // block sums in a fixed tree order
    constexpr int NK = PASS == 0 ? 6 : PASS == 1 ? 17 : PASS == 2 ? 4 : 21;
#pragma unroll
    for (int k = 0; k < NK; k++) {
        red[threadIdx.x] = acc[k];
        __syncthreads();
        for (int o = FIT_THREADS / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[size_t(blockIdx.x) * FIT_K + k] = red[0];
        __syncthreads();
    }
}

// sums the block partials (block order) and forms the pass's result
template <int PASS>
__global__ void k_fit_finish(FitInput in, const double* __restrict__ partial, FitState* __restrict__ st,
                             gls_raw_nlf* __restrict__ out) {
    __shared__ double tot[FIT_K];
    const int k = threadIdx.x;
    if (k < FIT_K) {
        double t = 0.0;
        for (int b = 0; b < FIT_BLOCKS; b++) t += partial[size_t(b) * FIT_K + k];
        tot[k] = t;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int n = nch(in);
    if (PASS == 0) {  // the variance bound from the class histogram
        const double* h = tot;
        const double b = h[0] > 1e3 ? 1.0e-5 : h[1] > 1e3 ? 1.0e-4 : h[2] > 1e3 ? 1.0e-3
                       : h[3] > 1e3 ? 1.0e-2 : h[4] > 1e3 ? 1.0e-1 : 1.0;
        for (int c = 0; c < 4; c++) st->bound[c] = b;
    } else if (PASS == 1) {
        const double N = tot[16];
        for (int c = 0; c < n; c++) {
            const double sx = tot[c], sy = tot[4 + c], sxx = tot[8 + c], sxy = tot[12 + c];
            st->B[c] = max_s((N * sxy - sx * sy) / (N * sxx - sx * sx), 1e-8);
            st->A[c] = max_s((sy - st->B[c] * sx) / N, 1e-8);
        }
        st->N1 = N;
    } else if (PASS == 2) {
        for (int c = 0; c < n; c++) {
            st->err2[c] = tot[c] / st->N1;
            st->bound[c] = st->B[c];  // the second pass keeps variances under the fitted slope
        }
    } else {
        const double N = tot[16];
        double newErr2[4];
        bool better = true, nan = false;
        for (int c = 0; c < n; c++) {
            newErr2[c] = tot[17 + c] / N;
            nan = nan || isnan(newErr2[c]);
            better = better && (in.raw ? newErr2[c] < st->err2[c] : newErr2[c] <= st->err2[c]);
        }
        const bool accept = in.raw ? (N > 0.001 * in.pixels && !nan && better) : (better && N / in.pixels > 0.01);
        double A[4], B[4];
        for (int c = 0; c < n; c++) {
            A[c] = st->A[c];
            B[c] = st->B[c];
            if (accept) {
                const double sx = tot[c], sy = tot[4 + c], sxx = tot[8 + c], sxy = tot[12 + c];
                B[c] = max_s((N * sxy - sx * sy) / (N * sxx - sx * sx), 1e-8);
                A[c] = max_s((sy - B[c] * sx) / N, 1e-8);
            }
        }
        const double adj = double(__fmul_rn(in.exposure, in.exposure));  // a float product, as in the reference
        for (int c = 0; c < 4; c++) {
            out->a[c] = c < n ? float(A[c] * adj) : 0.f;
            out->b[c] = c < n ? float(B[c] * adj) : 0.f;
        }
    }
}

void launch_fit(const FitInput& in, double* partial, FitState* st, gls_raw_nlf* out, cudaStream_t s) {
    k_fit_pass<0><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, st, partial);
    k_fit_finish<0><<<1, 32, 0, s>>>(in, partial, st, out);
    k_fit_pass<1><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, st, partial);
    k_fit_finish<1><<<1, 32, 0, s>>>(in, partial, st, out);
    k_fit_pass<2><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, st, partial);
    k_fit_finish<2><<<1, 32, 0, s>>>(in, partial, st, out);
    k_fit_pass<3><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, st, partial);
    k_fit_finish<3><<<1, 32, 0, s>>>(in, partial, st, out);
}

}  // namespace

size_t nlf_scratch_bytes() { return size_t(FIT_BLOCKS) * FIT_K * sizeof(double) + sizeof(FitState) + 64; }

template <class S>
int launch_measure_raw_nlf(Plane<S, 1> scaled, int pattern, Plane<float, 4> mean, Plane<float, 4> var,
                           float exposure, void* scratch, gls_raw_nlf* out, cudaStream_t s) {
    const dim3 g((mean.w + RS_TX - 1) / RS_TX, (mean.h + RS_TY - 1) / RS_TY);
    k_raw_stats<S><<<g, dim3(RS_TX, RS_TY), 0, s>>>(scaled, pattern, mean, var);
    FitInput in{reinterpret_cast<const float4*>(mean.p), reinterpret_cast<const float4*>(var.p), mean.w, mean.h,
                mean.pitch / 4, 1, double(scaled.w) * double(scaled.h), exposure};
    double* partial = static_cast<double*>(scratch);
    FitState* st = reinterpret_cast<FitState*>(partial + size_t(FIT_BLOCKS) * FIT_K);
    launch_fit(in, partial, st, out, s);
    return 9;
}

template <class S>
int launch_measure_ycc_nlf(Plane<S, 4> img, Plane<float, 4> stats, float exposure, void* scratch,
                           gls_raw_nlf* out, cudaStream_t s) {
    const dim3 g((img.w + YS_TX - 1) / YS_TX, (img.h + YS_TY - 1) / YS_TY);
    k_ycc_stats<S><<<g, dim3(YS_TX, YS_TY), 0, s>>>(img, stats);
    FitInput in{reinterpret_cast<const float4*>(stats.p), nullptr, stats.w, stats.h, stats.pitch / 4, 0,
                double(img.w) * double(img.h), exposure};
    double* partial = static_cast<double*>(scratch);
    FitState* st = reinterpret_cast<FitState*>(partial + size_t(FIT_BLOCKS) * FIT_K);
    launch_fit(in, partial, st, out, s);
    return 9;
}

template int launch_measure_raw_nlf<float>(Plane<float, 1>, int, Plane<float, 4>, Plane<float, 4>, float, void*,
                                           gls_raw_nlf*, cudaStream_t);
template int launch_measure_raw_nlf<__half>(Plane<__half, 1>, int, Plane<float, 4>, Plane<float, 4>, float, void*,
                                            gls_raw_nlf*, cudaStream_t);
template int launch_measure_ycc_nlf<float>(Plane<float, 4>, Plane<float, 4>, float, void*, gls_raw_nlf*,
                                           cudaStream_t);
template int launch_measure_ycc_nlf<__half>(Plane<__half, 4>, Plane<float, 4>, float, void*, gls_raw_nlf*,
                                            cudaStream_t);

}  // namespace gls
