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
// (325, indexed by pca_tri_index) then sum p (25). A block stages a
// chunk at a time in shared memory, converted to FP64 once per value; a
// thread issues all of its loads of a round before it stores any (the
// rounds are latency-bound: a few loads per thread, from L2). Its threads
// own the 350 accumulators (thread t the ones t, t + blockDim, ...), each
// summed patch by patch in four partial sums (patch k of the row into sum
// k mod 4), so a row's bits do not depend on the block size or the
// staging. The rows are summed in order by the eigen-solve, so the result
// does not depend on scheduling (no atomics).
constexpr int PC_CHUNK = kPcaChunk;
constexpr int PC_STAGE = PC_CHUNK;                           // patches staged per round
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
    // patch index -> (column, row) of the patch grid by a multiply-high:
    // q = umulhi(p, floor((2^32 - 1) / gw) + 1) is p / gw exactly while
    // p * gw < 2^32 (every frame up to ~100 MP); a division otherwise
    const bool fast_div = gw > 1 && uint64_t(n) * uint64_t(gw) < (1ull << 32);
    const uint32_t gmul = fast_div ? 0xffffffffu / uint32_t(gw) + 1u : 0u;
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
                    const int k = i / kPcaDim, e = i - k * kPcaDim;  // constant divisors
                    const int pidx = base + k;
                    const int prow = fast_div ? int(__umulhi(uint32_t(pidx), gmul)) : pidx / gw;
                    const int ey = e / 5;
                    const int px = (pidx - prow * gw) * 8 + (e - ey * 5) - 2, py = prow * 8 + ey - 2;
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
//      reflector steps, each a column norm, the product p = beta A v (a
//      thread per row), and the rank-2 update of the trailing block by all
//      threads (matrix in shared memory);
//   2. the 8 largest eigenvalues of T by Sturm-sequence multisection:
//      warp w brackets eigenvalue 24 - w (ascending order); its 32 lanes
//      count the eigenvalues below 32 points of the bracket, which shrinks
//      33-fold per round (7 rounds: 2.4e-11 of the spectrum width);
//   3. each eigenvector of T by inverse iteration: the tridiagonal
//      T - lambda I is factored once with partial pivoting (lane 0 of the
//      eigenvalue's warp) and solved three times from a start vector of its
//      own; tiny pivots are raised to eps ||T|| so the solve stays finite;
//   4. the back-transform z = H_0 (H_1 (... H_22 y)), one reflector at a
//      time for all 8 vectors (a thread per dot product, then the block),
//      and Gram-Schmidt of the 8 vectors in eigenvalue order, the classical
//      form applied twice (exactly equal eigenvalues give an orthonormal
//      basis of their eigenspace; distinct ones are already orthogonal).
//      FP64 warp shuffles are slow on this part (about 15 lanes per SM per
//      cycle), so no step reduces across a warp's lanes.
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

// 1 / sqrt(x) to FP64 accuracy for normal x > 0: the hardware approximation
// refined by two steps of Newton's method on f(r) = 1 / r^2 - x,
// r <- r (3 - x r^2) / 2, each doubling the correct bits.
__device__ __forceinline__ double rsqrt_nr(double x) {
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double hx = 0.5 * x;
    r = r * fma(-hx * r, r, 1.5);
    return r * fma(-hx * r, r, 1.5);
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

// sum_{i in [i0, i1)} a[i * sa] * b[i * sb] in four interleaved partial
// FP64 chains (i - i0 mod 4), added in a fixed order: a quarter of the
// latency of one chain
__device__ __forceinline__ double dot4(const double* a, int sa, const double* b, int sb, int i0, int i1) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int i = i0;
    for (; i + 4 <= i1; i += 4) {
        s0 = fma(a[i * sa], b[i * sb], s0);
        s1 = fma(a[(i + 1) * sa], b[(i + 1) * sb], s1);
        s2 = fma(a[(i + 2) * sa], b[(i + 2) * sb], s2);
        s3 = fma(a[(i + 3) * sa], b[(i + 3) * sb], s3);
    }
    if (i < i1) s0 = fma(a[i * sa], b[i * sb], s0);
    if (i + 1 < i1) s1 = fma(a[(i + 1) * sa], b[(i + 1) * sb], s1);
    if (i + 2 < i1) s2 = fma(a[(i + 2) * sa], b[(i + 2) * sb], s2);
    return (s0 + s1) + (s2 + s3);
}

struct EigenSmem {
    double acc[kPcaAcc];
    double A[EJ_N][EJ_N + 1];       // covariance, reduced in place
    double V[EJ_N - 2][EJ_N];       // Householder vectors (zero above k + 1)
    double beta[EJ_N - 2], vk1[EJ_N - 2];
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

    // ---- 1. Householder tridiagonalisation. Per step: thread 0 forms the
    //         reflector from column k (a sequential FP64 norm); thread j > k
    //         forms p_j = beta sum_i A[j][i] v_i; every thread forms
    //         K = (beta / 2) p.v and updates its entries of the trailing
    //         block, A' -= v w^T + w v^T with w = p - K v. v is column k below
    //         the diagonal with its first entry replaced (vk1), read from A
    //         itself; column k is outside every later trailing block.
    for (int k = 0; k < EJ_N - 2; k++) {
        if (t == 0) {
            // the norm and 1 / (v.v / 2) by refined hardware approximations:
            // the IEEE square root and division are long serial sequences
            // on this single thread's path
            const double nrm2 = dot4(&sm.A[0][k], EJ_N + 1, &sm.A[0][k], EJ_N + 1, k + 1, EJ_N);
            const double x1 = sm.A[k + 1][k];
            const bool skip = !(nrm2 > 1e-280);
            const double nrm = skip ? 0.0 : nrm2 * rsqrt_nr(nrm2);
            const double alpha = x1 >= 0.0 ? -nrm : nrm;
            const double den = nrm2 - alpha * x1;  // v.v / 2 > 0 unless the column is zero
            sm.beta[k] = skip ? 0.0 : rcp_nr(den);
            sm.vk1[k] = skip ? 0.0 : x1 - alpha;
            sm.d[k] = sm.A[k][k];
            sm.e[k] = skip ? x1 : alpha;
        }
        __syncthreads();
        const double beta = sm.beta[k];
        if (t < EJ_N) sm.V[k][t] = beta == 0.0 || t <= k ? 0.0 : (t == k + 1 ? sm.vk1[k] : sm.A[t][k]);
        if (beta == 0.0) continue;  // uniform: the column is already reduced
        const double v1 = sm.vk1[k];
        if (t > k && t < EJ_N)
            sm.p[t] = beta * fma(sm.A[t][k + 1], v1, dot4(&sm.A[t][0], 1, &sm.A[0][k], EJ_N + 1, k + 2, EJ_N));
        __syncthreads();
        const double K = 0.5 * beta * fma(sm.p[k + 1], v1, dot4(sm.p, 1, &sm.A[0][k], EJ_N + 1, k + 2, EJ_N));
        const int m = EJ_N - k - 1;
        for (int q = t; q < m * m; q += nth) {
            const int i = k + 1 + q / m, j = k + 1 + q % m;
            const double vi = i == k + 1 ? v1 : sm.A[i][k], vj = j == k + 1 ? v1 : sm.A[j][k];
            const double wi = sm.p[i] - K * vi, wj = sm.p[j] - K * vj;
            sm.A[i][j] -= vi * wj + wi * vj;
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
            const double inv = mx > 1e-290 && mx < 1e300 ? rcp_nr(mx) : 0.0;
            for (int i = 0; i < EJ_N; i++) y[i] *= inv;
        }
    }
    __syncthreads();
    // ---- 4. back-transform z = H_0 (H_1 (... H_22 y)), one reflector at a
    //         time for the 8 vectors: thread c forms the dot product of
    //         reflector k with vector c (a sequential FP64 chain, no warp
    //         reduction), then the block updates the vectors
    for (int k = EJ_N - 3; k >= 0; k--) {
        if (sm.beta[k] == 0.0) continue;  // uniform: the reflector is the identity
        if (t < EJ_TOP) sm.p[t] = sm.beta[k] * dot4(sm.V[k], 1, sm.y[t], 1, k + 1, EJ_N);  // V[k][i] = 0 for i <= k
        __syncthreads();
        for (int q = t; q < EJ_TOP * EJ_N; q += nth) {
            const int c = q / EJ_N, i = q % EJ_N;
            if (i > k) sm.y[c][i] -= sm.p[c] * sm.V[k][i];
        }
        __syncthreads();
    }
    // ---- 5. Gram-Schmidt in eigenvalue order, classical, twice per vector
    //         (as stable as the modified form): the dot products of vector c
    //         with the earlier ones by c threads at once, then the update by
    //         row; exactly equal eigenvalues give an orthonormal basis of
    //         their eigenspace, distinct ones are already orthogonal
    for (int c = 0; c < EJ_TOP; c++) {
        for (int pass = 0; pass < 2; pass++) {
            if (c == 0) break;
            if (t < c) sm.w[t] = dot4(sm.y[t], 1, sm.y[c], 1, 0, EJ_N);
            __syncthreads();
            if (t < EJ_N) {
                double v = sm.y[c][t];
                for (int k2 = 0; k2 < c; k2++) v -= sm.w[k2] * sm.y[k2][t];
                sm.y[c][t] = v;
            }
            __syncthreads();
        }
        if (t == 0) {
            const double nn = dot4(sm.y[c], 1, sm.y[c], 1, 0, EJ_N);
            const bool ok = nn > 1e-290 && nn < 1e300;
            sm.w[EJ_TOP] = ok ? rsqrt_nr(nn) : 0.0;
            if (!ok) sm.bad = 1;
        }
        __syncthreads();
        if (t < EJ_N) sm.y[c][t] = sm.w[EJ_TOP] != 0.0 ? sm.y[c][t] * sm.w[EJ_TOP] : 0.0;  // a non-finite vector is zeroed
        __syncthreads();
    }
    for (int q = t; q < EJ_TOP * EJ_N; q += nth) sm.Z[q % EJ_N][q / EJ_N] = sm.y[q / EJ_N][q % EJ_N];
    __syncthreads();
    // ---- 6. select_pca_basis. When every eigenvalue is kept (the usual
    //         case) it reduces to signing each column by its largest-magnitude
    //         entry (first on ties): thread c scans column c, then the block
    //         writes the basis, with the same result
    const double lam0 = sm.lam[0] > 0.0 ? sm.lam[0] : 0.0;
    bool all_kept = lam0 > 0.0;
    for (int c = 0; c < EJ_TOP; c++) all_kept = all_kept && sm.lam[c] > 1e-9 * lam0;
    if (all_kept) {
        if (t < EJ_TOP) {
            int amax = 0;
            for (int r = 1; r < EJ_N; r++)
                if (fabs(sm.y[t][r]) > fabs(sm.y[t][amax])) amax = r;
            sm.w[t] = sm.y[t][amax] < 0 ? -1.0 : 1.0;
        }
        __syncthreads();
        for (int q = t; q < EJ_N * EJ_TOP; q += nth) {
            const int r = q / EJ_TOP, c = q % EJ_TOP;
            basis[q] = float(sm.y[c][r] * sm.w[c]);
        }
    } else if (t == 0) {
        double ev[EJ_TOP];
        for (int c = 0; c < EJ_TOP; c++) ev[c] = sm.lam[c];
        select_pca_basis(ev, &sm.Z[0][0], EJ_TOP + 1, sm.work, basis);
    }
    if (t == 0 && status) *status = sm.bad ? -1 : EJ_INV_ITERS;
}


}  // namespace gls
