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
// SelfAdjointEigenSolver, PCA.cpp:36), FP64, one block. Only the 8 largest
// eigenpairs are needed, so the solve is the tridiagonal route of Golub &
// Van Loan (Matrix Computations, 4th ed.): section 8.3.1 and the
// bisection / inverse-iteration methods of sections 8.4.1 and 8.2.2
// (the tred2 / tridiagonal bisection / tinvit sequence of EISPACK):
//   1. Householder tridiagonalisation, A = Q T Q^T, Q = H_0 ... H_22: 23
//      reflector steps, each a warp-reduced column norm, the product
//      p = beta A v (one warp per row), and the rank-2 update of the
//      trailing block by all threads (matrix in shared memory);
//   2. the 8 largest eigenvalues of T by Sturm-sequence multisection:
//      warp w brackets eigenvalue 24 - w (ascending order); its 32 lanes
//      count the eigenvalues below 32 points of the bracket, which shrinks
//      33-fold per round (11 rounds reach FP64 resolution);
//   3. each eigenvector of T by inverse iteration: the tridiagonal
//      T - lambda I is factored once with partial pivoting (lane 0 of the
//      eigenvalue's warp) and solved three times from a start vector of its
//      own; tiny pivots are raised to eps ||T|| so the solve stays finite;
//   4. the back-transform z = H_0 (H_1 (... H_22 y)) by the warp, one
//      reflector at a time, and modified Gram-Schmidt of the 8 vectors in
//      eigenvalue order (exactly equal eigenvalues give an orthonormal basis
//      of their eigenspace; distinct ones are already orthogonal).
// The top-8 eigenvectors (descending eigenvalue, each signed so its
// largest-magnitude entry is positive; eigenvalues <= 1e-9 of the largest
// completed as in select_pca_basis) are written as a row-major 25x8 FP32
// basis. Every reduction has a fixed order, so the result is deterministic.
// status receives the number of inverse-iteration solves per vector (3), or
// -1 when a vector came out non-finite (the basis is then still written).
constexpr int EJ_THREADS = 704;  // 22 warps: two partial sums per accumulator in the prologue
constexpr int EJ_N = 25, EJ_TOP = 8, EJ_INV_ITERS = 3, EJ_MSEC_ROUNDS = 11;

// 1 / x to FP64 accuracy: the hardware approximation refined by two
// Newton-Raphson steps r <- r + r (1 - x r), each doubling the correct bits.
__device__ __forceinline__ double rcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    double e = fma(-x, r, 1.0);
    r = fma(r, e, r);
    e = fma(-x, r, 1.0);
    return fma(r, e, r);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x: the
// signs of the pivots of T - x I (Sturm sequence); a pivot smaller than
// pivmin in magnitude is replaced by -pivmin.
__device__ __forceinline__ int sturm_count(const double* d, const double* ee, double x, double pivmin) {
    double q = d[0] - x;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
#pragma unroll 8
    for (int i = 1; i < EJ_N; i++) {
        q = fma(-ee[i - 1], rcp_nr(q), d[i] - x);
        if (fabs(q) < pivmin) q = -pivmin;
        cnt += q < 0.0;
    }
    return cnt;
}

struct EigenSmem {
    double acc[kPcaAcc];
    double A[EJ_N][EJ_N + 1];       // covariance, reduced in place
    double V[EJ_N - 2][EJ_N];       // Householder vectors (zero above k + 1)
    double beta[EJ_N - 2];
    double d[EJ_N], e[EJ_N], ee[EJ_N];
    double p[EJ_N], w[EJ_N];
    double lam[EJ_TOP];
    // inverse iteration, per eigenvector: the pivoted LU of T - lambda I
    double u0[EJ_TOP][EJ_N], u1[EJ_TOP][EJ_N], u2[EJ_TOP][EJ_N], l[EJ_TOP][EJ_N], ru0[EJ_TOP][EJ_N];
    double y[EJ_TOP][EJ_N];
    unsigned char piv[EJ_TOP][EJ_N];
    double Z[EJ_N][EJ_TOP + 1];     // eigenvectors of A, column c = the c-th largest
    double work[200];
    double part2[kPcaAcc];
    int bad;
};

__global__ void __launch_bounds__(EJ_THREADS) k_pca_eigen(const double* __restrict__ part, int n_blocks,
                                                         int n_patches, float* __restrict__ basis, int* status) {
    __shared__ EigenSmem sm;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;

    if (n_patches < 2) {
        for (int k = t; k < 25 * 8; k += blockDim.x) basis[k] = ((k / 8) == (k % 8)) ? 1.f : 0.f;
        if (t == 0 && status) *status = 0;
        return;
    }
    // ---- block partials summed in a fixed order: two halves of the block
    //      range per accumulator, eight loads in flight each, then added
    {
        const int h = t / kPcaAcc, a = t % kPcaAcc;  // h: 0 or 1 (t < 700)
        const int half = (n_blocks + 1) / 2;
        const int b0 = h == 0 ? 0 : half, b1 = h == 0 ? half : n_blocks;
        double v = 0.0;
        if (t < 2 * kPcaAcc) {
            int b = b0;
            for (; b + 8 <= b1; b += 8) {
                double x[8];
#pragma unroll
                for (int k = 0; k < 8; k++) x[k] = part[(b + k) * kPcaAcc + a];
#pragma unroll
                for (int k = 0; k < 8; k++) v += x[k];
            }
            for (; b < b1; b++) v += part[b * kPcaAcc + a];
            if (h == 1) sm.part2[a] = v;
        }
        if (t == 0) sm.bad = 0;
        __syncthreads();
        if (t < kPcaAcc) sm.acc[t] = v + sm.part2[t];
    }
    __syncthreads();
    // ---- covariance from raw moments, (sum pp^T - n m m^T) / (n - 1)
    for (int k = t; k < EJ_N * EJ_N; k += blockDim.x) {
        const int i = k / EJ_N, j = k % EJ_N;
        const int idx = pca_tri_index(min(i, j), max(i, j));
        const double n = double(n_patches);
        const double mi = sm.acc[325 + i] / n, mj = sm.acc[325 + j] / n;
        sm.A[i][j] = (sm.acc[idx] - n * mi * mj) / (n - 1.0);
    }
    __syncthreads();

    // ---- 1. Householder tridiagonalisation
    for (int k = 0; k < EJ_N - 2; k++) {
        if (warp == 0) {
            // v from column k below the diagonal: x = A[k+1..][k]
            const double x = (lane > k && lane < EJ_N) ? sm.A[lane][k] : 0.0;
            const double nrm2 = warp_sum(x * x);
            const double x1 = __shfl_sync(0xffffffffu, x, k + 1);
            const double nrm = sqrt(nrm2);
            const double alpha = x1 >= 0.0 ? -nrm : nrm;
            const double den = nrm2 - alpha * x1;  // v.v / 2 > 0 unless the column is zero
            const bool skip = !(nrm2 > 1e-280);
            const double v = skip ? 0.0 : (lane == k + 1 ? x1 - alpha : x);
            if (lane < EJ_N) sm.V[k][lane] = v;
            if (lane == 0) {
                sm.beta[k] = skip ? 0.0 : 1.0 / den;
                sm.d[k] = sm.A[k][k];
                sm.e[k] = skip ? x1 : alpha;
            }
        }
        __syncthreads();
        const double beta = sm.beta[k];
        if (beta == 0.0) continue;  // uniform: the column is already reduced
        // p = beta A' v, one warp per row j > k
        for (int j = k + 1 + warp; j < EJ_N; j += EJ_THREADS / 32) {
            const double pr = warp_sum(lane < EJ_N ? sm.A[j][lane] * sm.V[k][lane] : 0.0);
            if (lane == 0) sm.p[j] = beta * pr;
        }
        __syncthreads();
        if (warp == 0) {  // w = p - (beta/2)(p.v) v
            const double vj = lane > k && lane < EJ_N ? sm.V[k][lane] : 0.0;
            const double pj = lane > k && lane < EJ_N ? sm.p[lane] : 0.0;
            const double pv = warp_sum(pj * vj);
            if (lane > k && lane < EJ_N) sm.w[lane] = pj - 0.5 * beta * pv * vj;
        }
        __syncthreads();
        // A' -= v w^T + w v^T on the trailing block
        const int m = EJ_N - k - 1;
        for (int q = t; q < m * m; q += blockDim.x) {
            const int i = k + 1 + q / m, j = k + 1 + q % m;
            sm.A[i][j] -= sm.V[k][i] * sm.w[j] + sm.w[i] * sm.V[k][j];
        }
        __syncthreads();
    }
    if (t == 0) {
        sm.d[EJ_N - 2] = sm.A[EJ_N - 2][EJ_N - 2];
        sm.d[EJ_N - 1] = sm.A[EJ_N - 1][EJ_N - 1];
        sm.e[EJ_N - 2] = sm.A[EJ_N - 1][EJ_N - 2];
        sm.e[EJ_N - 1] = 0.0;
    }
    __syncthreads();
    if (t < EJ_N) sm.ee[t] = sm.e[t] * sm.e[t];
    __syncthreads();

    // ---- 2. the 8 largest eigenvalues by Sturm multisection, warp w for
    //         eigenvalue index 24 - w (ascending)
    double tnorm = 0.0, lo = 0.0, hi = 0.0;
    {
        double a = 0.0, b = 0.0, s = 0.0;
        if (lane < EJ_N) {
            const double r = fabs(sm.e[lane]) + (lane > 0 ? fabs(sm.e[lane - 1]) : 0.0);
            a = sm.d[lane] - r;
            b = sm.d[lane] + r;
            s = fabs(sm.d[lane]) + r;
        } else {
            a = b = sm.d[0];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
            s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
        }
        tnorm = s;
        const double pad = 2.2e-16 * fmax(tnorm, 1e-300) * EJ_N;
        lo = a - pad;
        hi = b + pad;
    }
    const double pivmin = fmax(1e-290, 1e-290 * tnorm * tnorm);
    if (warp < EJ_TOP) {
        const int m = EJ_N - 1 - warp;
        for (int r = 0; r < EJ_MSEC_ROUNDS; r++) {
            if (!(hi - lo > 4.4e-16 * fmax(fabs(lo), fabs(hi)) + pivmin)) break;  // warp-uniform
            const double x = lo + (hi - lo) * (double(lane + 1) / 33.0);
            const int c = sturm_count(sm.d, sm.ee, x, pivmin);
            const unsigned above = __ballot_sync(0xffffffffu, c > m);
            const int first = above ? __ffs(above) - 1 : 32;
            const double xl = __shfl_sync(0xffffffffu, x, max(first - 1, 0));
            const double xh = __shfl_sync(0xffffffffu, x, min(first, 31));
            if (first > 0) lo = xl;
            if (first < 32) hi = xh;
        }
        if (lane == 0) sm.lam[warp] = 0.5 * (lo + hi);
    }
    __syncthreads();

    // ---- 3. inverse iteration on T for eigenvector `warp` (lane 0)
    if (warp < EJ_TOP && lane == 0) {
        const int c = warp;
        const double lam = sm.lam[c];
        const double tiny = fmax(2.2e-16 * tnorm, 1e-290);
        // factor T - lam I = P L U (Gaussian elimination, partial pivoting);
        // U has the diagonal u0 and two super-diagonals u1, u2
        double a = sm.d[0] - lam, b = sm.e[0];
        for (int k = 0; k < EJ_N - 1; k++) {
            const double cl = sm.e[k];                 // sub-diagonal entry of row k + 1
            const double an = sm.d[k + 1] - lam;       // diagonal of row k + 1
            const double bn = k + 1 < EJ_N - 1 ? sm.e[k + 1] : 0.0;
            if (fabs(a) >= fabs(cl)) {                 // no interchange
                double piv = a;
                if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
                const double rp = rcp_nr(piv);
                const double mult = cl * rp;
                sm.u0[c][k] = piv; sm.ru0[c][k] = rp; sm.u1[c][k] = b; sm.u2[c][k] = 0.0;
                sm.l[c][k] = mult; sm.piv[c][k] = 0;
                a = an - mult * b;
                b = bn;
            } else {                                   // rows k and k + 1 interchanged
                const double pc = fabs(cl) < tiny ? (cl < 0.0 ? -tiny : tiny) : cl;
                const double rp = rcp_nr(pc);
                const double mult = a * rp;
                sm.u0[c][k] = pc; sm.ru0[c][k] = rp; sm.u1[c][k] = an; sm.u2[c][k] = bn;
                sm.l[c][k] = mult; sm.piv[c][k] = 1;
                a = b - mult * an;
                b = -mult * bn;
            }
        }
        double piv = a;
        if (fabs(piv) < tiny) piv = piv < 0.0 ? -tiny : tiny;
        sm.u0[c][EJ_N - 1] = piv;
        sm.ru0[c][EJ_N - 1] = rcp_nr(piv);
        sm.u1[c][EJ_N - 1] = sm.u2[c][EJ_N - 1] = 0.0;
        // start vector of its own per eigenvector (deterministic)
        double* y = sm.y[c];
        for (int i = 0; i < EJ_N; i++) y[i] = 1.0 + 0.25 * double(((i + 1) * (7 + 4 * c)) % 13) / 13.0;
        for (int it = 0; it < EJ_INV_ITERS; it++) {
            for (int k = 0; k < EJ_N - 1; k++) {       // apply P and L^-1
                if (sm.piv[c][k]) {
                    const double tmp = y[k];
                    y[k] = y[k + 1];
                    y[k + 1] = tmp - sm.l[c][k] * y[k];
                } else {
                    y[k + 1] -= sm.l[c][k] * y[k];
                }
            }
            for (int k = EJ_N - 1; k >= 0; k--) {      // U^-1
                double s = y[k];
                if (k + 1 < EJ_N) s -= sm.u1[c][k] * y[k + 1];
                if (k + 2 < EJ_N) s -= sm.u2[c][k] * y[k + 2];
                y[k] = s * sm.ru0[c][k];
            }
            double mx = 0.0;                            // rescale by the largest entry
            for (int i = 0; i < EJ_N; i++) mx = fmax(mx, fabs(y[i]));
            const double inv = mx > 0.0 && mx < 1e300 ? 1.0 / mx : 0.0;
            for (int i = 0; i < EJ_N; i++) y[i] *= inv;
        }
    }
    __syncthreads();
    // ---- 4. back-transform by the reflectors (warp c, lane = row), then
    //         modified Gram-Schmidt in eigenvalue order (warp 0)
    if (warp < EJ_TOP) {
        const int c = warp;
        double z = lane < EJ_N ? sm.y[c][lane] : 0.0;
        for (int k = EJ_N - 3; k >= 0; k--) {
            const double vk = lane < EJ_N ? sm.V[k][lane] : 0.0;
            const double dot = warp_sum(vk * z);
            z -= sm.beta[k] * dot * vk;
        }
        if (lane < EJ_N) sm.Z[lane][c] = z;
    }
    __syncthreads();
    if (warp == 0) {
        for (int c = 0; c < EJ_TOP; c++) {
            double z = lane < EJ_N ? sm.Z[lane][c] : 0.0;
            for (int pass = 0; pass < 2; pass++)
                for (int k = 0; k < c; k++) {
                    const double zk = lane < EJ_N ? sm.Z[lane][k] : 0.0;
                    z -= warp_sum(zk * z) * zk;
                }
            const double nn = warp_sum(z * z);
            const bool ok = nn > 0.0 && nn < 1e300;
            z = ok ? z * (1.0 / sqrt(nn)) : 0.0;
            if (!ok && lane == 0) sm.bad = 1;
            if (lane < EJ_N) sm.Z[lane][c] = z;
            __syncwarp();
        }
        if (lane == 0) {
            double ev[EJ_TOP];
            for (int c = 0; c < EJ_TOP; c++) ev[c] = sm.lam[c];
            select_pca_basis(ev, &sm.Z[0][0], EJ_TOP + 1, sm.work, basis);
            if (status) *status = sm.bad ? -1 : EJ_INV_ITERS;
        }
    }
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
