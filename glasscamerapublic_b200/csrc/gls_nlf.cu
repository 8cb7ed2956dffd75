// gls_nlf.cu — noise-model measurement of RawConverter with
// calibrateFromImage:
//   * k_raw_stats    basicRawNoiseStatistics (demosaic.metal:1110-1136): the
//                    9x9 mean and variance of the four raw channels at every
//                    half-resolution position, from a shared-memory tile,
//                    and each position's variance class counted into the
//                    fit's histogram
//   * k_ycc_stats    basicNoiseStatistics (:1138-1159): the 5x5 mean of Y
//                    and variances of Y, Cb, Cr at every position of a
//                    level, and their variance classes
//   * k_fit_pass /   the two-pass least-squares fits of MeasureRawNLF
//     k_fit_finish   (raw_converter.cpp:339-490) and MeasureYCbCrNLF
//                    (pyramid_processor.cpp:173-324) on the device: each
//                    pass sums over the statistics in FP64 (fixed grid,
//                    block partial sums in a fixed order, so the result does
//                    not depend on scheduling) and a one-block kernel forms
//                    the fit from the partial sums
// The statistics are FP32 operation for operation as in the reference
// kernels (one rounding per operation, no contraction, each channel's taps
// in the reference's order), so the FP32 path's statistics equal the CPU
// oracle's bit for bit; the fits agree with the oracle's sequential FP64
// sums to their last bits.
#include <cmath>

#include "../../include/glscam.h"
#include "gls_common.cuh"
#include "gls_kernels.h"

namespace gls {

namespace {

// ---------------------------------------------------------------- statistics
// The variance class of a position: 6 + trunc(clamp(log10(v), -6, -1)) of
// its largest variance v (raw_converter.cpp:357-362), taken from the first
// channel on so that a NaN in a later channel never wins. The truncation
// makes the classes (0, 1e-6], (1e-6, 1e-5], (1e-5, 1e-4], (1e-4, 1e-3],
// (1e-3, 1e-2] and above; compared in FP64 on an FP32 variance, which lies
// more than 1e-11 (relative) from every power of ten, the thresholds give
// the logarithm's classes exactly. -1: no class (a NaN; for the YCbCr fit
// also a non-positive variance; a NaN largest value, which the reference
// turns into an undefined histogram index).
template <int N>
__device__ __forceinline__ int variance_class(const float (&v)[N], bool raw) {
    bool valid = true;
#pragma unroll
    for (int c = 0; c < N; c++) valid = valid && !isnan(v[c]) && (raw || v[c] > 0.f);
    if (!valid || v[0] < 0.f) return -1;  // log10 of a negative first variance is NaN
    float m = v[0];                        // 0: log10 = -inf, which any positive variance beats
#pragma unroll
    for (int c = 1; c < N; c++)
        if (v[c] > m) m = v[c];
    const double d = double(m);
    return d <= 1e-6 ? 0 : d <= 1e-5 ? 1 : d <= 1e-4 ? 2 : d <= 1e-3 ? 3 : d <= 1e-2 ? 4 : 5;
}

constexpr int RS_TX = 32, RS_TY = 8;                     // half-resolution positions per block
constexpr int RS_W = 2 * RS_TX + 10, RS_H = 2 * RS_TY + 10;  // full-resolution tile: 2x + [-4, 5]

// the block's class counts: a ballot per class in each warp, one shared
// atomic per warp and class
__device__ __forceinline__ void count_class(unsigned* cls, int k) {
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        const unsigned b = __ballot_sync(0xffffffffu, k == j);
        if (lane == 0 && b) atomicAdd(&cls[j], unsigned(__popc(b)));
    }
}

// PATTERN: the Bayer pattern, so every channel's tap set is known at
// compile time
template <class S, int PATTERN>
__global__ void __launch_bounds__(RS_TX* RS_TY) k_raw_stats(Plane<S, 1> raw, Plane<float, 4> mean,
                                                            Plane<float, 4> var, unsigned* __restrict__ hist) {
    constexpr int OX[4][4] = {{1, 0, 0, 1}, {0, 0, 1, 1}, {0, 0, 1, 1}, {1, 0, 0, 1}};
    constexpr int OY[4][4] = {{0, 0, 1, 1}, {1, 0, 0, 1}, {0, 1, 1, 0}, {1, 1, 0, 0}};
    __shared__ float tile[RS_H][RS_W];
    __shared__ unsigned cls[6];
    const int X0 = blockIdx.x * RS_TX, Y0 = blockIdx.y * RS_TY;  // half-resolution origin
    const int tid = threadIdx.y * RS_TX + threadIdx.x;
    if (tid < 6) cls[tid] = 0;
    for (int k = tid; k < RS_W * RS_H; k += RS_TX * RS_TY) {
        const int ty = k / RS_W, tx = k % RS_W;
        tile[ty][tx] = to_f(*raw.pxc(2 * X0 - 4 + tx, 2 * Y0 - 4 + ty));
    }
    __syncthreads();
    const int x = X0 + threadIdx.x, y = Y0 + threadIdx.y;
    int k = -1;
    if (x < mean.w && y < mean.h) {
        float sum[4] = {0.f, 0.f, 0.f, 0.f}, sumSq[4] = {0.f, 0.f, 0.f, 0.f};
        // the window steps one full-resolution pixel from 2 (x, y) - 4 and
        // reads each channel at its Bayer offset (readRAWQuad): channel c
        // reads the 10 x 10 block's 9 x 9 sub-block at its offset. Each
        // value is loaded once and added to the channels that read it, each
        // channel still in row-major order of its own taps.
        const int bx0 = 2 * threadIdx.x, by0 = 2 * threadIdx.y;
#pragma unroll
        for (int u = 0; u < 10; u++)
#pragma unroll
            for (int v = 0; v < 10; v++) {
                const float t = tile[by0 + u][bx0 + v];
                const float t2 = __fmul_rn(t, t);
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (u - OY[PATTERN][c] >= 0 && u - OY[PATTERN][c] < 9 && v - OX[PATTERN][c] >= 0 &&
                        v - OX[PATTERN][c] < 9) {
                        sum[c] = __fadd_rn(sum[c], t);
                        sumSq[c] = __fadd_rn(sumSq[c], t2);
                    }
            }
        f4 m, vv;
        float* mp = &m.x;
        float* vp = &vv.x;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            mp[c] = __fdiv_rn(sum[c], 81.f);
            vp[c] = __fdiv_rn(__fsub_rn(sumSq[c], __fdiv_rn(__fmul_rn(sum[c], sum[c]), 81.f)), 81.f);
        }
        st4<float>(mean.px(x, y), m);
        st4<float>(var.px(x, y), vv);
        const float vc[4] = {vv.x, vv.y, vv.z, vv.w};
        k = variance_class<4>(vc, true);
    }
    count_class(cls, k);
    __syncthreads();
    if (tid < 6 && cls[tid]) atomicAdd(&hist[tid], cls[tid]);
}

constexpr int YS_TX = 32, YS_TY = 8;
constexpr int YS_W = YS_TX + 4, YS_H = YS_TY + 4;

template <class S>
__global__ void __launch_bounds__(YS_TX* YS_TY) k_ycc_stats(Plane<S, 4> img, Plane<float, 4> stats,
                                                            unsigned* __restrict__ hist) {
    __shared__ float tile[3][YS_H][YS_W];
    __shared__ unsigned cls[6];
    const int x0 = blockIdx.x * YS_TX, y0 = blockIdx.y * YS_TY;
    const int tid = threadIdx.y * YS_TX + threadIdx.x;
    if (tid < 6) cls[tid] = 0;
    for (int k = tid; k < YS_W * YS_H; k += YS_TX * YS_TY) {
        const int ty = k / YS_W, tx = k % YS_W;
        const f4 p = ld4<S>(img.pxc(x0 - 2 + tx, y0 - 2 + ty));
        tile[0][ty][tx] = p.x;
        tile[1][ty][tx] = p.y;
        tile[2][ty][tx] = p.z;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    int k = -1;
    if (x < img.w && y < img.h) {
        float sum[3] = {0.f, 0.f, 0.f}, sumSq[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int dy = 0; dy < 5; dy++)
#pragma unroll
            for (int dx = 0; dx < 5; dx++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    const float t = tile[c][threadIdx.y + dy][threadIdx.x + dx];
                    sum[c] = __fadd_rn(sum[c], t);
                    sumSq[c] = __fadd_rn(sumSq[c], __fmul_rn(t, t));
                }
        f4 o;
        o.x = __fdiv_rn(sum[0], 25.f);
        float* op = &o.y;
#pragma unroll
        for (int c = 0; c < 3; c++)
            op[c] = __fdiv_rn(__fsub_rn(sumSq[c], __fdiv_rn(__fmul_rn(sum[c], sum[c]), 25.f)), 25.f);
        st4<float>(stats.px(x, y), o);
        const float vc[3] = {o.y, o.z, o.w};
        k = variance_class<3>(vc, false);
    }
    count_class(cls, k);
    __syncthreads();
    if (tid < 6 && cls[tid]) atomicAdd(&hist[tid], cls[tid]);
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

__device__ __forceinline__ Sample load_sample(const FitInput& in, long i) {
    const int x = int(i % in.w), y = int(i / in.w);
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

struct FitState {
    double bound[4];
    double A[4], B[4];
    double err2[4];
    double N1;
};

__device__ __forceinline__ double max_s(double v, double s) { return v > s ? v : s; }

// pass: 1 the first fit's sums; 2 its squared residuals; 3 the second fit's
// sums and squared residuals (the class histogram, pass 0, comes with the
// statistics)
template <int PASS>
__global__ void __launch_bounds__(FIT_THREADS) k_fit_pass(FitInput in, const FitState* __restrict__ st_,
                                                          double* __restrict__ partial) {
    constexpr int NK = PASS == 1 ? 17 : PASS == 2 ? 4 : 21;
    __shared__ double red[FIT_THREADS / 32][NK];
    double acc[NK];
#pragma unroll
    for (int k = 0; k < NK; k++) acc[k] = 0.0;
    const FitState st = *st_;
    const int n = nch(in);
    const long total = long(in.w) * in.h;
    for (long i = long(blockIdx.x) * FIT_THREADS + threadIdx.x; i < total; i += long(FIT_BLOCKS) * FIT_THREADS) {
        const Sample s = load_sample(in, i);
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
        } else if (PASS == 2) {
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c < n) {
                    const double d = (st.A[c] + st.B[c] * s.m[c]) - s.v[c];
                    acc[c] += d * d;
                }
        } else {
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
                        acc[17 + (c & 3)] += d2[c];
                    }
                acc[16] += 1.0;
            }
        }
    }
    // block sums in a fixed order: a shuffle tree per warp, then the warps
    // in order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NK; k++) {
        double v = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < NK) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < FIT_THREADS / 32; w++) t += red[w][threadIdx.x];
        partial[size_t(blockIdx.x) * FIT_K + threadIdx.x] = t;
    }
}

// sums the block partials (a warp per sum: lane-strided blocks, then a
// shuffle tree) and forms the pass's result; pass 0 forms the variance
// bound from the class histogram and leaves the histogram zeroed
template <int PASS>
__global__ void __launch_bounds__(FIT_K * 32) k_fit_finish(FitInput in, const double* __restrict__ partial,
                                                           unsigned* __restrict__ hist, FitState* __restrict__ st,
                                                           gls_raw_nlf* __restrict__ out) {
    __shared__ double tot[FIT_K];
    const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
    if (PASS > 0) {
        double v[(FIT_BLOCKS + 31) / 32];
#pragma unroll
        for (int j = 0; j < (FIT_BLOCKS + 31) / 32; j++) {  // every load issued before the sums
            const int b = lane + 32 * j;
            v[j] = b < FIT_BLOCKS ? partial[size_t(b) * FIT_K + k] : 0.0;
        }
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < (FIT_BLOCKS + 31) / 32; j++) t += v[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) tot[k] = t;
    } else if (threadIdx.x < 6) {
        tot[threadIdx.x] = double(hist[threadIdx.x]);
        hist[threadIdx.x] = 0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int n = nch(in);
    if (PASS == 0) {  // the variance bound from the class histogram (raw_converter.cpp:364-369)
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

struct FitScratch {
    double* partial;
    FitState* st;
    unsigned* hist;
};

FitScratch fit_scratch(void* scratch) {
    char* p = static_cast<char*>(scratch);
    FitScratch f;
    f.partial = reinterpret_cast<double*>(p);
    p += size_t(FIT_BLOCKS) * FIT_K * sizeof(double);
    f.st = reinterpret_cast<FitState*>(p);
    p += sizeof(FitState);
    f.hist = reinterpret_cast<unsigned*>(p);
    return f;
}

void launch_fit(const FitInput& in, const FitScratch& f, gls_raw_nlf* out, cudaStream_t s) {
    k_fit_finish<0><<<1, FIT_K * 32, 0, s>>>(in, f.partial, f.hist, f.st, out);
    k_fit_pass<1><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, f.st, f.partial);
    k_fit_finish<1><<<1, FIT_K * 32, 0, s>>>(in, f.partial, f.hist, f.st, out);
    k_fit_pass<2><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, f.st, f.partial);
    k_fit_finish<2><<<1, FIT_K * 32, 0, s>>>(in, f.partial, f.hist, f.st, out);
    k_fit_pass<3><<<FIT_BLOCKS, FIT_THREADS, 0, s>>>(in, f.st, f.partial);
    k_fit_finish<3><<<1, FIT_K * 32, 0, s>>>(in, f.partial, f.hist, f.st, out);
}

}  // namespace

// partial sums, the fit state and the class histogram (which each
// measurement leaves zeroed; zero the scratch when it is allocated)
size_t nlf_scratch_bytes() {
    return size_t(FIT_BLOCKS) * FIT_K * sizeof(double) + sizeof(FitState) + 8 * sizeof(unsigned);
}

template <class S>
int launch_measure_raw_nlf(Plane<S, 1> scaled, int pattern, Plane<float, 4> mean, Plane<float, 4> var,
                           float exposure, void* scratch, gls_raw_nlf* out, cudaStream_t s) {
    const FitScratch f = fit_scratch(scratch);
    const dim3 g((mean.w + RS_TX - 1) / RS_TX, (mean.h + RS_TY - 1) / RS_TY);
    const dim3 b(RS_TX, RS_TY);
    switch (pattern) {
        case 0: k_raw_stats<S, 0><<<g, b, 0, s>>>(scaled, mean, var, f.hist); break;
        case 1: k_raw_stats<S, 1><<<g, b, 0, s>>>(scaled, mean, var, f.hist); break;
        case 2: k_raw_stats<S, 2><<<g, b, 0, s>>>(scaled, mean, var, f.hist); break;
        default: k_raw_stats<S, 3><<<g, b, 0, s>>>(scaled, mean, var, f.hist); break;
    }
    FitInput in{reinterpret_cast<const float4*>(mean.p), reinterpret_cast<const float4*>(var.p), mean.w, mean.h,
                mean.pitch / 4, 1, double(scaled.w) * double(scaled.h), exposure};
    launch_fit(in, f, out, s);
    return 8;
}

template <class S>
int launch_measure_ycc_nlf(Plane<S, 4> img, Plane<float, 4> stats, float exposure, void* scratch,
                           gls_raw_nlf* out, cudaStream_t s) {
    const FitScratch f = fit_scratch(scratch);
    const dim3 g((img.w + YS_TX - 1) / YS_TX, (img.h + YS_TY - 1) / YS_TY);
    k_ycc_stats<S><<<g, dim3(YS_TX, YS_TY), 0, s>>>(img, stats, f.hist);
    FitInput in{reinterpret_cast<const float4*>(stats.p), nullptr, stats.w, stats.h, stats.pitch / 4, 0,
                double(img.w) * double(img.h), exposure};
    launch_fit(in, f, out, s);
    return 8;
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
