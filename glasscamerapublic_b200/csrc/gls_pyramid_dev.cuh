// gls_pyramid_dev.cuh — device code of one pyramid level shared by the
// stream kernels (gls_pyramid.cu) and the persistent batch kernel
// (gls_blockmatch.cu): a pixel of the reconstruct step, a covariance
// partial row, and the eigen-solve of the level's PCA basis. Both callers
// run the same code, so their results are bit-identical.
#pragma once

#include "gls_common.cuh"
#include "gls_kernels.h"
#include "gls_pca_pairs.h"

namespace gls {

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

// One pixel of subtractNoiseImage (demosaic.metal:922-959): the layer at
// (x, y) from the level's image, the coarse level's noisy and denoised
// images (bilinear, texel position ((x + 0.5) r - 0.5)) and the gradient.
template <class S>
__device__ __forceinline__ void subtract_noise_px(const Plane<S, 4>& in, const Plane<S, 4>& coarse,
                                                  const Plane<S, 4>& coarse_den, const Plane<S, 2>& grad,
                                                  const Plane<S, 4>& out, const SubtractArgs& a, float rx, float ry,
                                                  int x, int y) {
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
// the 5x5 luma neighbourhoods of (8x, 8y), x < W/8, y < H/8, taken in
// chunks of 64. Partial row r holds the FP64 sums over chunks
// [g r, g (r + 1)) (g chunks per row): the upper triangle of sum p p^T
// (325, indexed by pca_tri_index) then sum p (25). A block stages two
// chunks at a time in shared memory, converted to FP64 once per value; a
// thread issues all of its loads of a round before it stores any (the
// rounds are latency-bound: a few loads per thread, from L2). Its threads
// own the 350 accumulators (thread t the ones t, t + blockDim, ...), each
// summed patch by patch in four partial sums (patch k of the row into sum
// k mod 4), so a row's bits do not depend on the block size or the
// staging. The rows are summed in order by the eigen-solve, so the result
// does not depend on scheduling (no atomics).
constexpr int PC_CHUNK = kPcaChunk;
constexpr int PC_STAGE = 2 * PC_CHUNK;                       // patches staged per round
constexpr int PC_LOADS = (PC_STAGE * kPcaDim + 255) / 256;   // loads in flight per thread (256+ threads)

struct CovSmem {
    double sp[PC_STAGE][kPcaDim + 1];
};

template <class S>
__device__ __forceinline__ void pca_cov_row(Plane<S, 4> img, double* __restrict__ row, int chunk0, int chunk1,
                                            CovSmem& sm) {
    const int gw = img.w / 8, gh = img.h / 8;
    const int n = gw * gh;
    const int t = threadIdx.x, nth = blockDim.x;
    // four partial sums per accumulator (patches k = 0, 1, 2, 3 mod 4): FP64
    // chains a quarter as long; added in a fixed order at the end
    double sum[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
    int r[2] = {0, 0}, c[2] = {-1, -1};
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int a = t + j * nth;
        if (a < kPcaTri) pca_pair(a, r[j], c[j]);
        else if (a < kPcaAcc) r[j] = a - kPcaTri;
    }
    const int p_end = min(chunk1 * PC_CHUNK, n);
    for (int base = chunk0 * PC_CHUNK; base < p_end; base += PC_STAGE) {
        const int cnt = min(PC_STAGE, p_end - base);
        const int nv = cnt * kPcaDim;
        for (int i0 = 0; i0 < nv; i0 += PC_LOADS * nth) {
            float v[PC_LOADS];
#pragma unroll
            for (int u = 0; u < PC_LOADS; u++) {
                const int i = i0 + t + u * nth;
                v[u] = 0.f;
                if (i < nv) {
                    const int k = i / kPcaDim, e = i % kPcaDim;
                    const int pidx = base + k;
                    const int px = (pidx % gw) * 8 + (e % 5) - 2, py = (pidx / gw) * 8 + (e / 5) - 2;
                    v[u] = to_f(*img.pxc(px, py));
                }
            }
#pragma unroll
            for (int u = 0; u < PC_LOADS; u++) {
                const int i = i0 + t + u * nth;
                if (i < nv) sm.sp[i / kPcaDim][i % kPcaDim] = double(v[u]);
            }
        }
        __syncthreads();
        // patch k into partial sum k mod 4 (base is a multiple of 4, and cnt
        // is but in the last round of the level): products by FMA, the 25
        // component sums by additions
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int a = t + j * nth;
            if (a >= kPcaAcc) continue;
            const int rr = r[j], cc = c[j];
            double* s4 = sum[j];
            int k = 0;
            if (a < kPcaTri) {
                for (; k + 4 <= cnt; k += 4) {
#pragma unroll
                    for (int q = 0; q < 4; q++) s4[q] = fma(sm.sp[k + q][rr], sm.sp[k + q][cc], s4[q]);
                }
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (k + q < cnt) s4[q] = fma(sm.sp[k + q][rr], sm.sp[k + q][cc], s4[q]);
            } else {
                for (; k + 4 <= cnt; k += 4) {
#pragma unroll
                    for (int q = 0; q < 4; q++) s4[q] += sm.sp[k + q][rr];
                }
#pragma unroll
                for (int q = 0; q < 3; q++)
                    if (k + q < cnt) s4[q] += sm.sp[k + q][rr];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int a = t + j * nth;
        if (a < kPcaAcc) row[a] = ((sum[j][0] + sum[j][1]) + sum[j][2]) + sum[j][3];
    }
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
//      33-fold per round (7 rounds: 2.4e-11 of the spectrum width);
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
// 7 multisection rounds bracket each eigenvalue to 33^-7 (2.4e-11) of the
// spectrum's width: inverse iteration from such a shift converges in its
// three solves (the error shrinks by shift error / gap per solve), and the
// eigenvalue itself only orders the vectors and sets the rank threshold
constexpr int EJ_N = 25, EJ_TOP = 8, EJ_INV_ITERS = 3, EJ_MSEC_ROUNDS = 7;

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
    double part1[kPcaAcc], part2[kPcaAcc];
    int bad;
};

// The solve by one block of at least 8 warps (any size: every loop strides
// by the block size, and the bits do not depend on it).
__device__ inline void pca_eigen_block(const double* __restrict__ part, int n_blocks, int n_patches,
                                float* __restrict__ basis, int* status, EigenSmem& sm) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nth = blockDim.x;

    if (n_patches < 2) {
        for (int k = t; k < 25 * 8; k += nth) basis[k] = ((k / 8) == (k % 8)) ? 1.f : 0.f;
        if (t == 0 && status) *status = 0;
        return;
    }
    // ---- partial rows summed in a fixed order: two halves of the row range
    //      per accumulator, sixteen loads in flight each, then added
    {
        const int half = (n_blocks + 1) / 2;
        for (int q = t; q < 2 * kPcaAcc; q += nth) {
            const int h = q / kPcaAcc, a = q % kPcaAcc;
            const int b0 = h == 0 ? 0 : half, b1 = h == 0 ? half : n_blocks;
            double v = 0.0;
            int b = b0;
            for (; b + 16 <= b1; b += 16) {  // sixteen loads in flight
                double x[16];
#pragma unroll
                for (int k = 0; k < 16; k++) x[k] = part[size_t(b + k) * kPcaAcc + a];
#pragma unroll
                for (int k = 0; k < 16; k++) v += x[k];
            }
            for (; b < b1; b++) v += part[size_t(b) * kPcaAcc + a];
            (h == 0 ? sm.part1 : sm.part2)[a] = v;
        }
        if (t == 0) sm.bad = 0;
        __syncthreads();
        for (int a = t; a < kPcaAcc; a += nth) sm.acc[a] = sm.part1[a] + sm.part2[a];
    }
    __syncthreads();
    // ---- covariance from raw moments, (sum pp^T - n m m^T) / (n - 1)
    for (int k = t; k < EJ_N * EJ_N; k += nth) {
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
        for (int j = k + 1 + warp; j < EJ_N; j += nth / 32) {
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
        for (int q = t; q < m * m; q += nth) {
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
        // select_pca_basis; when every eigenvalue is kept (the usual case) it
        // reduces to signing each column by its largest-magnitude entry (first
        // on ties), done here by the warp, lane = row, with the same result
        const double lam0 = sm.lam[0] > 0.0 ? sm.lam[0] : 0.0;
        bool all_kept = lam0 > 0.0;
        for (int c = 0; c < EJ_TOP; c++) all_kept = all_kept && sm.lam[c] > 1e-9 * lam0;
        if (all_kept) {
            for (int c = 0; c < EJ_TOP; c++) {
                const double v = lane < EJ_N ? sm.Z[lane][c] : 0.0;
                double a = lane < EJ_N ? fabs(v) : -1.0;
                int idx = lane;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double a2 = __shfl_xor_sync(0xffffffffu, a, o);
                    const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
                    if (a2 > a || (a2 == a && i2 < idx)) {
                        a = a2;
                        idx = i2;
                    }
                }
                const double vmax = __shfl_sync(0xffffffffu, v, idx);
                const double sgn = vmax < 0 ? -1.0 : 1.0;
                if (lane < EJ_N) basis[lane * 8 + c] = float(v * sgn);
            }
        } else if (lane == 0) {
            double ev[EJ_TOP];
            for (int c = 0; c < EJ_TOP; c++) ev[c] = sm.lam[c];
            select_pca_basis(ev, &sm.Z[0][0], EJ_TOP + 1, sm.work, basis);
        }
        if (lane == 0 && status) *status = sm.bad ? -1 : EJ_INV_ITERS;
    }
}


}  // namespace gls
