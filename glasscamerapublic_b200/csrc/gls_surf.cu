// gls_surf.cu — registration and fusion on the GPU: RawChannels, the SURF
// integral image, fast-Hessian detector, orientation + 64-D descriptor,
// brute-force matching, RANSAC + least-squares homography, and the
// registerAndFuse / registerImage warps, behind the gls_surf_* / gls_*
// entry points of include/glscam.h.
//
// Reference: ImageRegistration/SURF.metal, SURF.cpp, Homography.cpp,
// LeastSquaresHomography.cpp, RTL/RANSAC.hpp, PyramidFusion/pyramidFusion.cpp.
// Every float expression that decides a keypoint, a descriptor or a model
// is evaluated with one IEEE rounding per operation (gls_fmath.h), so the
// results are bit-identical to the CPU restatement that checks them.
//
// Layout in HBM per detector: the integral image (W+1) x (H+1) F32 and its
// transposed column sums (W x H); 64000 candidate keypoints; per feature
// slot the kept keypoints (28 B) and descriptors (256 B). The detector
// computes Hessian determinants tile by tile in shared memory and runs the
// 3x3x3 non-maximum suppression on them in the same kernel, so no
// determinant plane is ever written to HBM.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <set>
#include <type_traits>
#include <vector>

#include "gls_common.cuh"
#include "gls_devbuf.h"
#include "gls_fmath.h"

namespace gls {

using glsm::dadd;
using glsm::ddiv;
using glsm::dmul;
using glsm::dsqrt;
using glsm::dsub;
using glsm::fadd;
using glsm::fdiv;
using glsm::fmul;
using glsm::fsqrt;
using glsm::fsub;
using glsm::gls_atan2f;
using glsm::gls_cosf;
using glsm::gls_sinf;

constexpr int kMaxKeypoints = GLS_SURF_MAX_KEYPOINTS;
constexpr int kMaxOctaves = 6;
constexpr int kLayers = 4;  // nOctaveLayers + 2 with nOctaveLayers = 2 (the only layer count served)

// ------------------------------------------------------------ host: patterns
struct Box {
    int x1, y1, x2, y2;
    float w;
};

// resizeHaarPattern (SURF.cpp:103-114)
template <int N>
static void resize_haar(const int src[][5], Box* dst, int old_size, int new_size) {
    const float ratio = float(new_size) / float(old_size);
    for (int k = 0; k < N; k++) {
        const int dx1 = int(std::lrint(ratio * float(src[k][0])));
        const int dy1 = int(std::lrint(ratio * float(src[k][1])));
        const int dx2 = int(std::lrint(ratio * float(src[k][2])));
        const int dy2 = int(std::lrint(ratio * float(src[k][3])));
        dst[k] = {dx1, dy1, dx2, dy2, float(src[k][4]) / (float(dx2 - dx1) * float(dy2 - dy1))};
    }
}

// One Hessian layer: the box corners the Metal kernel reads (gpuSurfHF,
// SURF.cpp:200-225) and its margin crop (DetAndTraceHaarPattern,
// SURF.cpp:235-265).
struct LayerDev {
    short dx[8][2];   // r02 r07 r32 r37 | r62 r67 r92 r97 (x, y)
    short dy[8][2];   // r20 r23 r70 r73 | r26 r76 r29 r79
    short dxy[4][4][2];
    float w, wxy;
    int mx, my, mw, mh;
    int size;
};

struct OctaveDev {
    LayerDev layer[kLayers];
    int step, lw, lh;      // layer grid = image / step
    int tiles_x, tiles_y;  // detector tiles over the layer grid
    int block0;            // first block of this octave
};

struct DetectArgs {
    OctaveDev oct[kMaxOctaves];
    int n_oct;
    const float* sum;
    int sum_pitch;  // floats
    float threshold;
    int per_axis;  // corrected interpolation (else the reference's scale-offset broadcast)
    gls_keypoint* cand;
    int* cand_count;
};

static LayerDev make_layer(int sum_w, int sum_h, int size, int step) {
    static const int dx_s[3][5] = {{0, 2, 3, 7, 1}, {3, 2, 6, 7, -2}, {6, 2, 9, 7, 1}};
    static const int dy_s[3][5] = {{2, 0, 7, 3, 1}, {2, 3, 7, 6, -2}, {2, 6, 7, 9, 1}};
    static const int dxy_s[4][5] = {{1, 1, 4, 4, 1}, {5, 1, 8, 4, -1}, {1, 5, 4, 8, -1}, {5, 5, 8, 8, 1}};
    Box bx[3], by[3], bxy[4];
    resize_haar<3>(dx_s, bx, 9, size);
    resize_haar<3>(dy_s, by, 9, size);
    resize_haar<4>(dxy_s, bxy, 9, size);
    LayerDev L{};
    auto set = [](short* d, int x, int y) {
        d[0] = short(x);
        d[1] = short(y);
    };
    set(L.dx[0], bx[0].x1, bx[0].y1);
    set(L.dx[1], bx[0].x1, bx[0].y2);
    set(L.dx[2], bx[0].x2, bx[0].y1);
    set(L.dx[3], bx[0].x2, bx[0].y2);
    set(L.dx[4], bx[1].x2, bx[1].y1);
    set(L.dx[5], bx[1].x2, bx[1].y2);
    set(L.dx[6], bx[2].x2, bx[2].y1);
    set(L.dx[7], bx[2].x2, bx[2].y2);
    set(L.dy[0], by[0].x1, by[0].y1);
    set(L.dy[1], by[0].x1, by[0].y2);
    set(L.dy[2], by[0].x2, by[0].y1);
    set(L.dy[3], by[0].x2, by[0].y2);
    set(L.dy[4], by[1].x1, by[1].y2);
    set(L.dy[5], by[1].x2, by[1].y2);
    set(L.dy[6], by[2].x1, by[2].y2);
    set(L.dy[7], by[2].x2, by[2].y2);
    for (int k = 0; k < 4; k++) {
        set(L.dxy[k][0], bxy[k].x1, bxy[k].y1);
        set(L.dxy[k][1], bxy[k].x1, bxy[k].y2);
        set(L.dxy[k][2], bxy[k].x2, bxy[k].y1);
        set(L.dxy[k][3], bxy[k].x2, bxy[k].y2);
    }
    L.w = bx[0].w;
    L.wxy = bxy[0].w;
    L.mx = (size / 2) / step;
    L.my = (size / 2) / step;
    L.mw = 1 + (sum_w - 1 - size) / step;
    L.mh = 1 + (sum_h - 1 - size) / step;
    if (size > sum_w - 1 || size > sum_h - 1) L.mw = L.mh = 0;  // the wavelet does not fit: no samples
    L.size = size;
    return L;
}

// ------------------------------------------------------------ device: Hessian
__device__ __forceinline__ float rect_gpu(float tr, float tl, float br, float bl) {
    return fsub(fadd(0.5f, fsub(tr, tl)), fsub(br, bl));
}

// calcHaarPatternDx / Dy / Dxy + calcDetAndTrace (SURF.metal:77-145)
__device__ __forceinline__ void det_trace_at(const float* __restrict__ S, int pitch, int px, int py,
                                             const LayerDev& L, float* det, float* trace) {
    auto rd = [&](const short* o) { return __ldg(S + size_t(py + o[1]) * pitch + px + o[0]); };
    const float r02 = rd(L.dx[0]), r07 = rd(L.dx[1]), r32 = rd(L.dx[2]), r37 = rd(L.dx[3]);
    const float r62 = rd(L.dx[4]), r67 = rd(L.dx[5]), r92 = rd(L.dx[6]), r97 = rd(L.dx[7]);
    const float dx = fmul(L.w, fsub(rect_gpu(r97, r92, r07, r02), fmul(3.0f, rect_gpu(r67, r62, r37, r32))));
    const float r20 = rd(L.dy[0]), r23 = rd(L.dy[1]), r70 = rd(L.dy[2]), r73 = rd(L.dy[3]);
    const float r26 = rd(L.dy[4]), r76 = rd(L.dy[5]), r29 = rd(L.dy[6]), r79 = rd(L.dy[7]);
    const float dy = fmul(L.w, fsub(rect_gpu(r79, r70, r29, r20), fmul(3.0f, rect_gpu(r76, r73, r26, r23))));
    float dxy = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float wk = (k == 0 || k == 3) ? L.wxy : -L.wxy;
        const float p0 = rd(L.dxy[k][0]), p1 = rd(L.dxy[k][1]), p2 = rd(L.dxy[k][2]), p3 = rd(L.dxy[k][3]);
        dxy = fadd(dxy, fmul(wk, rect_gpu(p0, p1, p2, p3)));
    }
    *det = fsub(fmul(dx, dy), fmul(fmul(0.81f, dxy), dxy));
    *trace = fadd(dx, dy);
}

__device__ __forceinline__ float det3(const float a[3], const float b[3], const float c[3]) {
    const float cx = fsub(fmul(b[1], c[2]), fmul(b[2], c[1]));
    const float cy = fsub(fmul(b[2], c[0]), fmul(b[0], c[2]));
    const float cz = fsub(fmul(b[0], c[1]), fmul(b[1], c[0]));
    return fadd(fadd(fmul(a[0], cx), fmul(a[1], cy)), fmul(a[2], cz));
}

constexpr int DT_X = 32, DT_Y = 8;  // NMS positions per detector tile

// A feature slot's count, set from a host value (gls_surf_load_features).
__global__ void k_store_count(int* count, int n) { *count = n; }

// calcDetAndTrace for the four layers of an octave over a tile plus a
// one-sample halo, into shared memory; then findMaximaInLayer
// (SURF.metal:249-313) with interpolateKeypoint (:207-247) for the two
// middle layers. Determinants outside a layer's margin crop are 0, as an
// unwritten determinant plane.
__global__ void __launch_bounds__(256) k_hessian_nms(DetectArgs a) {
    __shared__ float det[kLayers][DT_Y + 2][DT_X + 2];
    int o = 0;
    while (o + 1 < a.n_oct && int(blockIdx.x) >= a.oct[o + 1].block0) o++;
    const OctaveDev& O = a.oct[o];
    const int b = blockIdx.x - O.block0;
    const int bx = b % O.tiles_x, by = b / O.tiles_x;
    const int x0 = bx * DT_X, y0 = by * DT_Y;
    const int step = O.step;
    for (int i = threadIdx.x; i < kLayers * (DT_Y + 2) * (DT_X + 2); i += blockDim.x) {
        const int l = i / ((DT_Y + 2) * (DT_X + 2));
        const int r = i % ((DT_Y + 2) * (DT_X + 2));
        const int ly = r / (DT_X + 2), lx = r % (DT_X + 2);
        const int gx = x0 + lx - 1, gy = y0 + ly - 1;
        const LayerDev& L = O.layer[l];
        const int ix = gx - L.mx, iy = gy - L.my;
        float d = 0.0f;
        if (ix >= 0 && ix < L.mw && iy >= 0 && iy < L.mh) {
            float t;
            det_trace_at(a.sum, a.sum_pitch, ix * step, iy * step, L, &d, &t);
        }
        det[l][ly][lx] = d;
    }
    __syncthreads();
    const int tx = threadIdx.x % DT_X, ty = threadIdx.x / DT_X;
    const int x = x0 + tx, y = y0 + ty;
#pragma unroll
    for (int l = 1; l <= 2; l++) {
        const LayerDev& L = O.layer[l];
        const int margin = (O.layer[l + 1].size / 2) / step + 1;
        if (x < margin || x >= O.lw - margin || y < margin || y >= O.lh - margin) continue;
        const float v = det[l][ty + 1][tx + 1];
        if (!(v > a.threshold)) continue;
        bool mx = true;
        for (int i = 0; i < 3 && mx; i++)
            for (int dy = -1; dy <= 1 && mx; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (i == 1 && dx == 0 && dy == 0) continue;
                    if (!(v > det[l - 1 + i][ty + 1 + dy][tx + 1 + dx])) {
                        mx = false;
                        break;
                    }
                }
        if (!mx) continue;
        auto n9 = [&](int i, int dy, int dx) { return det[l - 1 + i][ty + 1 + dy][tx + 1 + dx]; };
        const int size = L.size, s0 = O.layer[l - 1].size;
        const int sum_y = step * (y - (size / 2) / step);
        const int sum_x = step * (x - (size / 2) / step);
        float dtmp, tr = 0.0f;  // trace plane value; 0 outside the crop, as unwritten
        if (x - L.mx < L.mw && y - L.my < L.mh)
            det_trace_at(a.sum, a.sum_pitch, (x - L.mx) * step, (y - L.my) * step, L, &dtmp, &tr);
        gls_keypoint kp;
        kp.x = fadd(float(sum_x), fmul(float(size - 1), 0.5f));
        kp.y = fadd(float(sum_y), fmul(float(size - 1), 0.5f));
        kp.size = float(size);
        kp.angle = -1.0f;
        kp.response = v;
        kp.octave = o;
        kp.class_id = tr > 0.0f ? 1 : 0;
        const float B[3] = {-fdiv(fsub(n9(1, 0, 1), n9(1, 0, -1)), 2.0f), -fdiv(fsub(n9(1, 1, 0), n9(1, -1, 0)), 2.0f),
                            -fdiv(fsub(n9(2, 0, 0), n9(0, 0, 0)), 2.0f)};
        const float dxx = fadd(fsub(n9(1, 0, -1), fmul(2.0f, n9(1, 0, 0))), n9(1, 0, 1));
        const float dxy = fdiv(fadd(fsub(fsub(n9(1, 1, 1), n9(1, 1, -1)), n9(1, -1, 1)), n9(1, -1, -1)), 4.0f);
        const float dxs = fdiv(fadd(fsub(fsub(n9(2, 0, 1), n9(2, 0, -1)), n9(0, 0, 1)), n9(0, 0, -1)), 4.0f);
        const float dyy = fadd(fsub(n9(1, -1, 0), fmul(2.0f, n9(1, 0, 0))), n9(1, 1, 0));
        const float dys = fdiv(fadd(fsub(fsub(n9(2, 1, 0), n9(2, -1, 0)), n9(0, 1, 0)), n9(0, -1, 0)), 4.0f);
        const float dss = fadd(fsub(n9(0, 0, 0), fmul(2.0f, n9(1, 0, 0))), n9(2, 0, 0));
        const float A0[3] = {dxx, dxy, dxs}, A1[3] = {dxy, dyy, dys}, A2[3] = {dxs, dys, dss};
        float X[3] = {0.0f, 0.0f, 0.0f};
        const float dt = det3(A0, A1, A2);
        if (dt != 0.0f) {  // solve3x3 (SURF.metal:189-205)
            X[2] = fdiv(det3(A0, A1, B), dt);
            if (a.per_axis) {
                X[0] = fdiv(det3(B, A1, A2), dt);
                X[1] = fdiv(det3(A0, B, A2), dt);
            } else {  // `(float3)(a, b, c) / det` is float3(c) / det: the scale offset in every lane
                X[0] = X[1] = X[2];
            }
        }
        const bool all_zero = X[0] == 0.0f && X[1] == 0.0f && X[2] == 0.0f;
        if (all_zero || !(fabsf(X[0]) <= 1.0f && fabsf(X[1]) <= 1.0f && fabsf(X[2]) <= 1.0f)) continue;
        kp.x = fadd(kp.x, fmul(X[0], float(step)));
        kp.y = fadd(kp.y, fmul(X[1], float(step)));
        kp.size = rintf(fadd(kp.size, fmul(X[2], float(size - s0))));
        const int idx = atomicAdd(a.cand_count, 1);
        if (idx < kMaxKeypoints) a.cand[idx] = kp;
    }
}

// KeypointGreater (SURF.cpp:1215-1227), with the candidate index as the
// last key so that the order is total.
__device__ __forceinline__ bool kp_before(const gls_keypoint& a, int ia, const gls_keypoint& b, int ib) {
    if (a.response != b.response) return a.response > b.response;
    if (a.size != b.size) return a.size > b.size;
    if (a.octave != b.octave) return a.octave > b.octave;
    if (a.y != b.y) return a.y > b.y;
    if (a.x != b.x) return a.x < b.x;
    return ia < ib;
}

// Rank sort of the candidates and the max_features cut (SURF.cpp:1285,
// 1413-1418): candidate i goes to its rank if the rank is below keep.
__global__ void __launch_bounds__(256) k_keypoint_rank(const gls_keypoint* __restrict__ cand,
                                                       const int* __restrict__ cand_count, int keep,
                                                       gls_keypoint* __restrict__ out, int* __restrict__ out_count) {
    __shared__ gls_keypoint tile[256];
    const int n = min(*cand_count, kMaxKeypoints);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x >= n) return;  // whole block past the end (block-uniform)
    gls_keypoint me{};
    if (i < n) me = cand[i];
    int rank = 0;
    for (int j0 = 0; j0 < n; j0 += 256) {
        __syncthreads();
        if (j0 + threadIdx.x < n) tile[threadIdx.x] = cand[j0 + threadIdx.x];
        __syncthreads();
        const int m = min(256, n - j0);
        if (i < n)
            for (int j = 0; j < m; j++) rank += kp_before(tile[j], j0 + j, me, i) ? 1 : 0;
    }
    if (i < n && rank < keep) out[rank] = me;
    if (i == 0) *out_count = min(n, keep);
}

// ------------------------------------------------------------ descriptors
struct DescTables {  // SURFInvoker constructor (SURF.cpp:466-497)
    float apt_x[169], apt_y[169], aptw[169];
    float dw[400];
    int n_ori;
};

__device__ __forceinline__ float rect_cpu(float tr, float tl, float br, float bl) {
    // SURF.cpp:79-82: the 0.5 is a double literal
    return __double2float_rn(dsub(dadd(0.5, double(fsub(tr, tl))), double(fsub(br, bl))));
}

// calcHaarPattern (SURF.cpp:84-101) over two boxes
__device__ __forceinline__ float haar2(const float* __restrict__ S, int pitch, int px, int py, const Box* f) {
    float d = 0.0f;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const Box& b = f[k];
        const float p0 = __ldg(S + size_t(py + b.y1) * pitch + px + b.x1);
        const float p1 = __ldg(S + size_t(py + b.y2) * pitch + px + b.x1);
        const float p2 = __ldg(S + size_t(py + b.y1) * pitch + px + b.x2);
        const float p3 = __ldg(S + size_t(py + b.y2) * pitch + px + b.x2);
        d = fadd(d, fmul(b.w, rect_cpu(p0, p1, p2, p3)));
    }
    return d;
}

__device__ void resize_haar2_dev(const int (*src)[5], Box* dst, int new_size) {
    const float ratio = fdiv(float(new_size), 4.0f);
    for (int k = 0; k < 2; k++) {
        const int dx1 = lrintf(fmul(ratio, float(src[k][0])));
        const int dy1 = lrintf(fmul(ratio, float(src[k][1])));
        const int dx2 = lrintf(fmul(ratio, float(src[k][2])));
        const int dy2 = lrintf(fmul(ratio, float(src[k][3])));
        dst[k] = {dx1, dy1, dx2, dy2, fdiv(float(src[k][4]), fmul(float(dx2 - dx1), float(dy2 - dy1)))};
    }
}

struct DescArgs {
    const float* img;
    int img_pitch, iw, ih;
    const float* sum;
    int sum_pitch, sw, sh;
    const DescTables* tab;
    gls_keypoint* kps;
    const int* count;
    float* desc;
    int all;  // describe every keypoint (else the reference's ranges, SURF.cpp:681-693)
};

constexpr int kDescThreads = 128;
constexpr int kMaxWinIdx = 42;  // rows / columns of the window resizeVV reads

// SURFInvoker::computeRange for one keypoint per block (SURF.cpp:499-677):
// dominant orientation over the Haar responses in a radius-6s disc, the
// rotated window (only the 42 x 42 of its pixels that resizeVV reads,
// each at the position the reference's running sums reach), the 21 x 21
// patch, 20 x 20 gradients and the 4 x 4 x 4 descriptor.
__global__ void __launch_bounds__(kDescThreads) k_describe(DescArgs a) {
    const int k = blockIdx.x;
    const int n = *a.count;
    if (k >= n) return;
    // SURFInvoker::run cuts K > 32 keypoints into ceil(K/8) ranges of
    // ceil(K/8): the first min(K, ceil(K/8)^2) are described, the others keep
    // angle -1 and a zero descriptor
    const int r8 = (n + 7) / 8;
    if (!a.all && n > 32 && k >= r8 * r8) {
        for (int i = threadIdx.x; i < 64; i += blockDim.x) a.desc[size_t(k) * 64 + i] = 0.0f;
        return;
    }
    __shared__ float X[169], Y[169], ANG[169];
    __shared__ int pos[169];
    __shared__ float bx_s[72], by_s[72], mod_s[72];
    __shared__ float rowx[kMaxWinIdx], rowy[kMaxWinIdx];
    __shared__ int q[kMaxWinIdx];
    __shared__ float M[kMaxWinIdx][kMaxWinIdx + 1];
    __shared__ float P[21][22];
    __shared__ float DX[20][21], DY[20][21];
    __shared__ float cell[16][4];
    __shared__ Box dxt[2], dyt[2];
    __shared__ int nangle_s;
    __shared__ float dir_s;
    const DescTables& T = *a.tab;
    const int t = threadIdx.x;
    gls_keypoint kp = a.kps[k];
    float* desc = a.desc + size_t(k) * 64;
    for (int i = t; i < 64; i += blockDim.x) desc[i] = 0.0f;
    const float s = fdiv(fmul(kp.size, 1.2f), 9.0f);
    const int gws = 2 * lrintf(fmul(2.0f, s));
    if (a.sh < gws || a.sw < gws) {
        if (t == 0) a.kps[k].size = -1.0f;
        return;
    }
    if (t == 0) {
        const int dx_s[2][5] = {{0, 0, 2, 4, -1}, {2, 0, 4, 4, 1}};
        const int dy_s[2][5] = {{0, 0, 4, 2, 1}, {0, 2, 4, 4, -1}};
        resize_haar2_dev(dx_s, dxt, gws);
        resize_haar2_dev(dy_s, dyt, gws);
    }
    __syncthreads();
    // orientation samples, compacted in the reference's sample order
    const float half_wav = fdiv(float(gws - 1), 2.0f);
    int valid[2] = {0, 0};
    float vxs[2], vys[2];
    for (int r = 0; r < 2; r++) {
        const int kk = t + r * kDescThreads;
        if (kk >= T.n_ori) continue;
        const int x = lrintf(fsub(fadd(kp.x, fmul(T.apt_x[kk], s)), half_wav));
        const int y = lrintf(fsub(fadd(kp.y, fmul(T.apt_y[kk], s)), half_wav));
        if (y < 0 || y >= a.sh - gws || x < 0 || x >= a.sw - gws) continue;
        vxs[r] = haar2(a.sum, a.sum_pitch, x, y, dxt);
        vys[r] = haar2(a.sum, a.sum_pitch, x, y, dyt);
        valid[r] = 1;
    }
    for (int r = 0; r < 2; r++) {
        const int kk = t + r * kDescThreads;
        if (kk < 169) pos[kk] = (kk < T.n_ori) ? valid[r] : 0;
    }
    __syncthreads();
    if (t == 0) {  // exclusive scan over at most 169 flags
        int acc = 0;
        for (int i = 0; i < T.n_ori; i++) {
            const int v = pos[i];
            pos[i] = acc;
            acc += v;
        }
        nangle_s = acc;
    }
    __syncthreads();
    for (int r = 0; r < 2; r++) {
        const int kk = t + r * kDescThreads;
        if (kk >= T.n_ori || !valid[r]) continue;
        const int j = pos[kk];
        const float xv = fmul(vxs[r], T.aptw[kk]), yv = fmul(vys[r], T.aptw[kk]);
        X[j] = xv;
        Y[j] = yv;
        const float tdeg = __double2float_rn(dmul(double(gls_atan2f(yv, xv)), 180.0 / 3.14159265358979323846));
        ANG[j] = tdeg < 0.0f ? fadd(tdeg, 360.0f) : tdeg;
    }
    __syncthreads();
    const int nangle = nangle_s;
    if (nangle == 0) {
        if (t == 0) a.kps[k].size = -1.0f;
        return;
    }
    if (t < 72) {
        const float bin = float(5 * t);
        float sx = 0.0f, sy = 0.0f;
        for (int j = 0; j < nangle; j++) {
            const float d = fabsf(fsub(float(lrintf(ANG[j])), bin));
            if (d < 30.0f || d > 330.0f) {
                sx = fadd(sx, X[j]);
                sy = fadd(sy, Y[j]);
            }
        }
        bx_s[t] = sx;
        by_s[t] = sy;
        mod_s[t] = fadd(fmul(sx, sx), fmul(sy, sy));
    }
    __syncthreads();
    if (t == 0) {  // the first bin with the largest modulus above 0
        float best = 0.0f, bestx = 0.0f, besty = 0.0f;
        for (int b = 0; b < 72; b++)
            if (mod_s[b] > best) {
                best = mod_s[b];
                bestx = bx_s[b];
                besty = by_s[b];
            }
        dir_s = gls_atan2f(-besty, bestx);
        a.kps[k].angle = dir_s;
    }
    __syncthreads();
    const float dir = fmul(dir_s, float(3.14159265358979323846 / 180.0));
    const float sin_dir = -gls_sinf(dir);
    const float cos_dir = gls_cosf(dir);
    const int win = int(fmul(21.0f, s));
    const float dsize = fdiv(float(win), 21.0f);
    if (t < 21) {
        const int qi = int(fmul(float(t), dsize));
        q[2 * t] = qi;
        q[2 * t + 1] = qi + 1;
    }
    __syncthreads();
    if (t == 0) {  // row starts: the running sums of the window's outer loop
        const float off = -fdiv(float(win - 1), 2.0f);
        float sx = fadd(fadd(kp.x, fmul(off, cos_dir)), fmul(off, sin_dir));
        float sy = fadd(fsub(kp.y, fmul(off, sin_dir)), fmul(off, cos_dir));
        int need = 0;
        for (int r = 0; need < kMaxWinIdx && r <= q[kMaxWinIdx - 1]; r++) {
            while (need < kMaxWinIdx && q[need] == r) {
                rowx[need] = sx;
                rowy[need] = sy;
                need++;
            }
            sx = fadd(sx, sin_dir);
            sy = fadd(sy, cos_dir);
        }
    }
    __syncthreads();
    if (t < kMaxWinIdx) {  // one requested window row per thread
        const int ncols1 = a.iw - 1, nrows1 = a.ih - 1;
        float px = rowx[t], py = rowy[t];
        int need = 0;
        for (int c = 0; need < kMaxWinIdx && c <= q[kMaxWinIdx - 1]; c++) {
            if (q[need] == c) {
                const int ix = int(floorf(px)), iy = int(floorf(py));
                float v;
                if (unsigned(ix) < unsigned(ncols1) && unsigned(iy) < unsigned(nrows1)) {
                    const float fa = fsub(px, float(ix)), fb = fsub(py, float(iy));
                    const float oa = fsub(1.0f, fa), ob = fsub(1.0f, fb);
                    const float* r0 = a.img + size_t(iy) * a.img_pitch;
                    const float* r1 = r0 + a.img_pitch;
                    const float top = fadd(fmul(__ldg(r0 + ix), oa), fmul(__ldg(r0 + ix + 1), fa));
                    const float bot = fadd(fmul(__ldg(r1 + ix), oa), fmul(__ldg(r1 + ix + 1), fa));
                    v = roundf(fadd(fmul(top, ob), fmul(bot, fb)));
                } else {
                    const int xx = min(max(int(roundf(px)), 0), ncols1);
                    const int yy = min(max(int(roundf(py)), 0), nrows1);
                    v = __ldg(a.img + size_t(yy) * a.img_pitch + xx);
                }
                while (need < kMaxWinIdx && q[need] == c) M[t][need++] = v;
            }
            px = fadd(px, cos_dir);
            py = fsub(py, sin_dir);
        }
    }
    __syncthreads();
    for (int e = t; e < 441; e += blockDim.x) {  // resizeVV (SURF.cpp:427-446)
        const int i = e / 21, j = e % 21;
        const float fi = fmul(float(i), dsize), fj = fmul(float(j), dsize);
        const int ii = int(fi), jj = int(fj);
        const float id = fsub(fi, float(ii)), jd = fsub(fj, float(jj));
        float v = 0.0f;
        if (jj < win - 1 && ii < win - 1) {
            const float oi = fsub(1.0f, id), oj = fsub(1.0f, jd);
            v = fmul(fmul(oi, oj), M[2 * i][2 * j]);
            v = fadd(v, fmul(fmul(id, oj), M[2 * i + 1][2 * j]));
            v = fadd(v, fmul(fmul(jd, oi), M[2 * j][2 * j + 1]));
            v = fadd(v, fmul(fmul(id, jd), M[2 * i + 1][2 * j + 1]));
        }
        P[i][j] = v;
    }
    __syncthreads();
    for (int e = t; e < 400; e += blockDim.x) {
        const int i = e / 20, j = e % 20;
        const float dw = T.dw[e];
        DX[i][j] = fmul(fsub(fadd(fsub(P[i][j + 1], P[i][j]), P[i + 1][j + 1]), P[i + 1][j]), dw);
        DY[i][j] = fmul(fsub(fadd(fsub(P[i + 1][j], P[i][j]), P[i + 1][j + 1]), P[i][j + 1]), dw);
    }
    __syncthreads();
    if (t < 16) {
        const int ci = t / 4, cj = t % 4;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
        for (int y = ci * 5; y < ci * 5 + 5; y++)
            for (int x = cj * 5; x < cj * 5 + 5; x++) {
                const float tx = DX[y][x], ty = DY[y][x];
                s0 = fadd(s0, tx);
                s1 = fadd(s1, ty);
                s2 = fadd(s2, fabsf(tx));
                s3 = fadd(s3, fabsf(ty));
            }
        cell[t][0] = s0;
        cell[t][1] = s1;
        cell[t][2] = s2;
        cell[t][3] = s3;
    }
    __syncthreads();
    __shared__ float scale_s;
    if (t == 0) {
        float sq = 0.0f;
        for (int c = 0; c < 16; c++)
            for (int m = 0; m < 4; m++) sq = fadd(sq, fmul(cell[c][m], cell[c][m]));
        scale_s = __double2float_rn(ddiv(1.0, double(fadd(fsqrt(sq), FLT_EPSILON))));
    }
    __syncthreads();
    if (t < 64) desc[t] = fmul(cell[t / 4][t % 4], scale_s);
}

// ------------------------------------------------------------ matching
// A batch of matching / homography jobs: each pairs a query slot (the
// reference frame's features) with a train slot; blockIdx.y is the job.
constexpr int kMaxJobs = 64;
struct MatchJob {
    const float* d1;
    const int* n1;
    const gls_keypoint* k1;
    const float* d2;
    const int* n2;
    const gls_keypoint* k2;
};
struct MatchJobs {
    MatchJob j[kMaxJobs];
};

// matchKeyPoints (SURF.metal:441-487): 24 lanes per query scan the train
// descriptors j = lane, lane + 24, ...; the L2 norm accumulates in four
// float lanes (SURF.metal:423-431). One warp per query.
__global__ void __launch_bounds__(128) k_match(MatchJobs jobs, int cap, gls_match* __restrict__ out_all) {
    const MatchJob& J = jobs.j[blockIdx.y];
    gls_match* out = out_all + size_t(blockIdx.y) * cap;
    const float* __restrict__ d1 = J.d1;
    const float* __restrict__ d2 = J.d2;
    const int lane = threadIdx.x & 31;
    const int i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int n1 = *J.n1, n2 = *J.n2;
    if (i >= n1) return;
    const float* p1 = d1 + size_t(i) * 64;
    float dmin = FLT_MAX;
    int jmin = 0;
    if (lane < 24) {
        for (int j = 0; j + lane < n2; j += 24) {
            const float4* p2 = reinterpret_cast<const float4*>(d2 + size_t(j + lane) * 64);
            const float4* q1 = reinterpret_cast<const float4*>(p1);
            float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
#pragma unroll 4
            for (int g = 0; g < 16; g++) {
                const float4 u = __ldg(q1 + g), v = __ldg(p2 + g);
                const float e0 = fsub(u.x, v.x), e1 = fsub(u.y, v.y), e2 = fsub(u.z, v.z), e3 = fsub(u.w, v.w);
                s0 = fadd(s0, fmul(e0, e0));
                s1 = fadd(s1, fmul(e1, e1));
                s2 = fadd(s2, fmul(e2, e2));
                s3 = fadd(s3, fmul(e3, e3));
            }
            const float d = fsqrt(fadd(fadd(fadd(s0, s1), s2), s3));
            if (d < dmin) {
                dmin = d;
                jmin = j + lane;
            }
        }
    }
    // lane 0 takes the lanes in order, strictly smaller wins
    float best = __shfl_sync(0xffffffffu, dmin, 0);
    int bj = __shfl_sync(0xffffffffu, jmin, 0);
    for (int l = 1; l < 24; l++) {
        const float dl = __shfl_sync(0xffffffffu, dmin, l);
        const int jl = __shfl_sync(0xffffffffu, jmin, l);
        if (dl < best) {
            best = dl;
            bj = jl;
        }
    }
    if (lane == 0) out[i] = {i, bj, best};
}

// refineMatch order (SURF.cpp:917-929): distance, then query index; the
// sorted matches become point pairs (query pt, train pt) as findMatches
// builds them (SURF.hpp:65-75).
__global__ void __launch_bounds__(256) k_match_rank(MatchJobs jobs, int cap, const gls_match* __restrict__ m_all,
                                                    gls_match* __restrict__ sorted_all, float4* __restrict__ pairs_all) {
    __shared__ gls_match tile[256];
    const MatchJob& J = jobs.j[blockIdx.y];
    const gls_match* __restrict__ m = m_all + size_t(blockIdx.y) * cap;
    gls_match* __restrict__ sorted = sorted_all + size_t(blockIdx.y) * cap;
    float4* __restrict__ pairs = pairs_all + size_t(blockIdx.y) * cap;
    const gls_keypoint* __restrict__ k1 = J.k1;
    const gls_keypoint* __restrict__ k2 = J.k2;
    const int n = *J.n1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x >= n) return;
    gls_match me{};
    if (i < n) me = m[i];
    int rank = 0;
    for (int j0 = 0; j0 < n; j0 += 256) {
        __syncthreads();
        if (j0 + threadIdx.x < n) tile[threadIdx.x] = m[j0 + threadIdx.x];
        __syncthreads();
        const int c = min(256, n - j0);
        if (i < n)
            for (int j = 0; j < c; j++) {
                const gls_match& o = tile[j];
                rank += (o.distance < me.distance || (o.distance == me.distance && o.query_idx < me.query_idx)) ? 1 : 0;
            }
    }
    if (i < n) {
        sorted[rank] = me;
        const gls_keypoint a = k1[me.query_idx], b = k2[me.train_idx];
        pairs[rank] = make_float4(a.x, a.y, b.x, b.y);
    }
}

// ------------------------------------------------------------ homography
// FindLeastSquaresHomography (LeastSquaresHomography.cpp:355-423) with the
// Jacobi solver of :218-353; hypot(p, q) is sqrt(p^2 + q^2). One warp
// solves one system: the rotations of a Jacobi step update disjoint element
// pairs, one pair per lane, so the warp produces the sequential loop's
// results bit for bit.
__device__ __forceinline__ double hypot_d(double a, double b) { return dsqrt(dadd(dmul(a, a), dmul(b, b))); }

constexpr unsigned kFull = 0xffffffffu;

struct LsWarp {  // shared scratch of one warp
    double a[81], V[81], W[9], T[9];
    double cen[4], mad[4];  // (cm0, cm1, cM0, cM1) and (sm0, sm1, sM0, sM1)
    double nrm[4][4];       // the 4 sample points, normalised (a0, a1, b0, b1)
    int indR[9], indC[9];
};

__device__ __forceinline__ void jac_rot(double& v0, double& v1, double c, double s) {
    const double a0 = v0, b0 = v1;
    v0 = dsub(dmul(a0, c), dmul(b0, s));
    v1 = dadd(dmul(a0, s), dmul(b0, c));
}

// column m > k of the largest |a[k][m]| (the first on ties)
__device__ __forceinline__ int max_in_row(const double* a, int k) {
    int m = k + 1;
    double mv = fabs(a[k * 9 + m]);
    for (int i = k + 2; i < 9; i++) {
        const double val = fabs(a[k * 9 + i]);
        if (mv < val) mv = val, m = i;
    }
    return m;
}

// row m < k of the largest |a[m][k]| (the first on ties)
__device__ __forceinline__ int max_in_col(const double* a, int k) {
    int m = 0;
    double mv = fabs(a[k]);
    for (int i = 1; i < k; i++) {
        const double val = fabs(a[i * 9 + k]);
        if (mv < val) mv = val, m = i;
    }
    return m;
}

// Jacobi eigen-solve of the symmetric S.a (destroyed): eigenvalues S.W
// sorted descending, eigenvectors as the rows of S.V. Called by a whole warp.
__device__ void jacobi9_warp(LsWarp& S) {
    constexpr int N = 9;
    const int lane = threadIdx.x & 31;
    double* a = S.a;
    if (lane < N) {
        for (int i = 0; i < N; i++) S.V[lane * N + i] = i == lane ? 1.0 : 0.0;
        S.W[lane] = a[lane * N + lane];
        if (lane < N - 1) S.indR[lane] = max_in_row(a, lane);
        if (lane > 0) S.indC[lane] = max_in_col(a, lane);
    }
    __syncwarp();
    for (int it = 0; it < N * N * 30; it++) {
        int k = 0, l = 0, stop = 0;
        double c = 0.0, s = 0.0;
        if (lane == 0) {
            double mv = fabs(a[S.indR[0]]);
            for (int i = 1; i < N - 1; i++) {
                const double val = fabs(a[i * N + S.indR[i]]);
                if (mv < val) mv = val, k = i;
            }
            l = S.indR[k];
            for (int i = 1; i < N; i++) {
                const double val = fabs(a[S.indC[i] * N + i]);
                if (mv < val) mv = val, k = S.indC[i], l = i;
            }
            const double p = a[k * N + l];
            if (fabs(p) <= DBL_EPSILON) {
                stop = 1;
            } else {
                const double y = dmul(dsub(S.W[l], S.W[k]), 0.5);
                double t = dadd(fabs(y), hypot_d(p, y));
                s = hypot_d(p, t);
                c = ddiv(t, s);
                s = ddiv(p, s);
                t = dmul(ddiv(p, t), p);
                if (y < 0) {
                    s = -s;
                    t = -t;
                }
                a[k * N + l] = 0.0;
                S.W[k] = dsub(S.W[k], t);
                S.W[l] = dadd(S.W[l], t);
            }
        }
        stop = __shfl_sync(kFull, stop, 0);
        if (stop) break;
        k = __shfl_sync(kFull, k, 0);
        l = __shfl_sync(kFull, l, 0);
        c = __shfl_sync(kFull, c, 0);
        s = __shfl_sync(kFull, s, 0);
        __syncwarp();
        if (lane < N) {  // k < l always: indR points right, indC points up
            if (lane != k && lane != l) {
                if (lane < k) jac_rot(a[lane * N + k], a[lane * N + l], c, s);
                else if (lane < l) jac_rot(a[k * N + lane], a[lane * N + l], c, s);
                else jac_rot(a[k * N + lane], a[l * N + lane], c, s);
            }
            jac_rot(S.V[k * N + lane], S.V[l * N + lane], c, s);
        }
        __syncwarp();
        if (lane < 2) {
            const int idx = lane == 0 ? k : l;
            if (idx < N - 1) S.indR[idx] = max_in_row(a, idx);
            if (idx > 0) S.indC[idx] = max_in_col(a, idx);
        }
        __syncwarp();
    }
    if (lane == 0) {
        for (int k = 0; k < N - 1; k++) {
            int m = k;
            for (int i = k + 1; i < N; i++)
                if (S.W[m] < S.W[i]) m = i;
            if (k != m) {
                const double tw = S.W[m];
                S.W[m] = S.W[k];
                S.W[k] = tw;
                for (int i = 0; i < N; i++) {
                    const double tv = S.V[m * N + i];
                    S.V[m * N + i] = S.V[k * N + i];
                    S.V[k * N + i] = tv;
                }
            }
        }
    }
    __syncwarp();
}

// entry j of the rows Lx, Ly of LeastSquaresHomography.cpp:396-397
__device__ __forceinline__ double lx_entry(int j, double a0, double a1, double b0) {
    switch (j) {
        case 0: return a0;
        case 1: return a1;
        case 2: return 1.0;
        case 6: return dmul(-b0, a0);
        case 7: return dmul(-b0, a1);
        case 8: return -b0;
        default: return 0.0;
    }
}
__device__ __forceinline__ double ly_entry(int j, double a0, double a1, double b1) {
    switch (j) {
        case 3: return a0;
        case 4: return a1;
        case 5: return 1.0;
        case 6: return dmul(-b1, a0);
        case 7: return dmul(-b1, a1);
        case 8: return -b1;
        default: return 0.0;
    }
}

// upper-triangle entry e (0..44) -> (j, k), j <= k
__device__ __forceinline__ void tri_index(int e, int& j, int& k) {
    j = 0;
    while (e >= 9 - j) {
        e -= 9 - j;
        j++;
    }
    k = j + e;
}

// The tail of the normalised DLT on S.a (full symmetric LtL), S.cen and
// S.mad: least eigenvector, de-normalisation, scale to H[2][2] = 1. Warp.
__device__ void ls_finish_warp(LsWarp& S, float* H) {
    const int lane = threadIdx.x & 31;
    jacobi9_warp(S);
    const double* h0 = &S.V[72];
    const double cm0 = S.cen[0], cm1 = S.cen[1], cM0 = S.cen[2], cM1 = S.cen[3];
    const double sm0 = S.mad[0], sm1 = S.mad[1], sM0 = S.mad[2], sM1 = S.mad[3];
    if (lane < 9) {
        const double inv[9] = {sm0, 0, cm0, 0, sm1, cm1, 0, 0, 1};
        const int i = lane / 3, j = lane % 3;
        double acc = 0.0;
        for (int k = 0; k < 3; k++) acc = dadd(acc, dmul(inv[i * 3 + k], h0[k * 3 + j]));
        S.T[lane] = acc;
    }
    __syncwarp();
    double r = 0.0;
    if (lane < 9) {
        const double nrm[9] = {ddiv(1.0, sM0), 0, ddiv(-cM0, sM0), 0, ddiv(1.0, sM1), ddiv(-cM1, sM1), 0, 0, 1};
        const int i = lane / 3, j = lane % 3;
        for (int k = 0; k < 3; k++) r = dadd(r, dmul(S.T[i * 3 + k], nrm[k * 3 + j]));
    }
    const double r8 = __shfl_sync(kFull, r, 8);
    if (lane < 9) H[lane] = fdiv(__double2float_rn(r), __double2float_rn(r8));
    __syncwarp();
}

// The 4-point model of one RANSAC sample; false where the reference throws
// (a degenerate spread). Warp.
__device__ bool ls4_warp(LsWarp& S, const float4* __restrict__ P, const int* __restrict__ idx, float* H) {
    const int lane = threadIdx.x & 31;
    auto comp = [](const float4& p, int c) { return c == 0 ? p.z : c == 1 ? p.w : c == 2 ? p.x : p.y; };
    if (lane < 4) {
        double acc = 0.0;
        for (int i = 0; i < 4; i++) acc = dadd(acc, double(comp(P[idx[i]], lane)));
        S.cen[lane] = ddiv(acc, 4.0);
    }
    __syncwarp();
    if (lane < 4) {
        double acc = 0.0;
        for (int i = 0; i < 4; i++) acc = dadd(acc, fabs(dsub(double(comp(P[idx[i]], lane)), S.cen[lane])));
        S.mad[lane] = ddiv(acc, 4.0);
    }
    __syncwarp();
    const double eps = DBL_EPSILON;
    if (fabs(S.mad[0]) < eps || fabs(S.mad[1]) < eps || fabs(S.mad[2]) < eps || fabs(S.mad[3]) < eps) return false;
    if (lane < 4) {
        const float4 p = P[idx[lane]];
        S.nrm[lane][0] = ddiv(dsub(double(p.x), S.cen[2]), S.mad[2]);
        S.nrm[lane][1] = ddiv(dsub(double(p.y), S.cen[3]), S.mad[3]);
        S.nrm[lane][2] = ddiv(dsub(double(p.z), S.cen[0]), S.mad[0]);
        S.nrm[lane][3] = ddiv(dsub(double(p.w), S.cen[1]), S.mad[1]);
    }
    __syncwarp();
    for (int e = lane; e < 45; e += 32) {
        int j, k;
        tri_index(e, j, k);
        double acc = 0.0;
        for (int q = 0; q < 4; q++) {
            const double* v = S.nrm[q];
            const double xj = lx_entry(j, v[0], v[1], v[2]), xk = lx_entry(k, v[0], v[1], v[2]);
            const double yj = ly_entry(j, v[0], v[1], v[3]), yk = ly_entry(k, v[0], v[1], v[3]);
            acc = dadd(acc, dadd(dmul(xj, xk), dmul(yj, yk)));
        }
        S.a[j * 9 + k] = acc;
        S.a[k * 9 + j] = acc;  // completeSymm
    }
    __syncwarp();
    ls_finish_warp(S, H);
    return true;
}

// applyHomography + squared error (Homography.cpp:65-70)
__device__ __forceinline__ float h_error(const float* H, float4 p) {
    const float w = fadd(fadd(fmul(H[6], p.x), fmul(H[7], p.y)), H[8]);
    const float u = fdiv(fadd(fadd(fmul(H[0], p.x), fmul(H[1], p.y)), H[2]), w);
    const float v = fdiv(fadd(fadd(fmul(H[3], p.x), fmul(H[4], p.y)), H[5]), w);
    const float dx = fsub(u, p.z), dy = fsub(v, p.w);
    return fadd(fmul(dx, dx), fmul(dy, dy));
}

// One RANSAC problem per job: its point pairs, their count and the sample
// table drawn for that count.
struct RansacJob {
    const float4* pairs;
    const int* samples;
    int n;
};
struct RansacJobs {
    RansacJob j[kMaxJobs];
};

// RANSAC hypotheses (RTL/RANSAC.hpp:47-66, 101-108): one warp per
// iteration fits its sample and counts the errors above the threshold.
constexpr int kHypWarps = 4;
__global__ void __launch_bounds__(32 * kHypWarps) k_ransac_models(RansacJobs jobs, int iters, float threshold,
                                                                  float* __restrict__ models_all,
                                                                  int* __restrict__ losses_all) {
    __shared__ LsWarp S[kHypWarps];
    __shared__ float Hs[kHypWarps][9];
    const RansacJob& J = jobs.j[blockIdx.y];
    const float4* __restrict__ pairs = J.pairs;
    const int* __restrict__ samples = J.samples;
    const int n = J.n;
    float* __restrict__ models = models_all + size_t(blockIdx.y) * iters * 9;
    int* __restrict__ losses = losses_all + size_t(blockIdx.y) * iters;
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int it = blockIdx.x * kHypWarps + w;
    if (it >= iters) return;  // warp-uniform
    float* H = Hs[w];
    if (!ls4_warp(S[w], pairs, samples + 4 * it, H)) {
        if (lane < 9) H[lane] = (lane % 4 == 0) ? 1.0f : 0.0f;
        __syncwarp();
    }
    int c = 0;
    for (int i = lane; i < n; i += 32) c += fabsf(h_error(H, pairs[i])) > threshold ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if (lane == 0) losses[it] = c;
    if (lane < 9) models[it * 9 + lane] = H[lane];
}

// The first model with the least loss, its inliers (|error| < threshold,
// in index order) and, with 4 or more, their least-squares refit
// (Homography.cpp:90-113). One block; the sequential sums read the inliers
// staged in shared memory.
constexpr int kFinalThreads = 256;
constexpr int kStage = 512;
__global__ void __launch_bounds__(kFinalThreads) k_ransac_final(RansacJobs jobs, int cap,
                                                                 const float* __restrict__ models_all,
                                                                 const int* __restrict__ losses_all, int iters,
                                                                 float threshold, int* __restrict__ inliers_all,
                                                                 int* __restrict__ n_inliers_all,
                                                                 float* __restrict__ H_all,
                                                                 float* __restrict__ loss_all) {
    const int job = blockIdx.x;
    const float4* __restrict__ pairs = jobs.j[job].pairs;
    const int n = jobs.j[job].n;
    const float* __restrict__ models = models_all + size_t(job) * iters * 9;
    const int* __restrict__ losses = losses_all + size_t(job) * iters;
    int* __restrict__ inliers = inliers_all + size_t(job) * cap;
    int* __restrict__ n_inliers = n_inliers_all + job;
    float* __restrict__ Hout = H_all + size_t(job) * 9;
    float* __restrict__ loss_out = loss_all + job;
    __shared__ int best_s, base_s;
    __shared__ float H[9], Hf[9];
    __shared__ int wsum[kFinalThreads / 32];
    __shared__ LsWarp S;
    __shared__ float4 stage[kStage];
    __shared__ double4 nstage[kStage];
    __shared__ double L[81];
    __shared__ int red_loss[kFinalThreads / 32], red_idx[kFinalThreads / 32];
    const int t = threadIdx.x;
    {  // the first iteration with the least loss: (loss, index) minimum
        int bl = INT_MAX, bi = INT_MAX;
        for (int i = t; i < iters; i += kFinalThreads) {
            const int v = losses[i];
            if (v < bl) bl = v, bi = i;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const int ol = __shfl_xor_sync(kFull, bl, o), oi = __shfl_xor_sync(kFull, bi, o);
            if (ol < bl || (ol == bl && oi < bi)) bl = ol, bi = oi;
        }
        if ((t & 31) == 0) {
            red_loss[t >> 5] = bl;
            red_idx[t >> 5] = bi;
        }
        __syncthreads();
        if (t == 0) {
            for (int w = 1; w < kFinalThreads / 32; w++)
                if (red_loss[w] < bl || (red_loss[w] == bl && red_idx[w] < bi)) bl = red_loss[w], bi = red_idx[w];
            best_s = bi;
            base_s = 0;
        }
    }
    __syncthreads();
    if (t < 9) H[t] = models[best_s * 9 + t];
    __syncthreads();
    for (int i0 = 0; i0 < n; i0 += kFinalThreads) {  // ordered compaction of the inliers
        const int i = i0 + t;
        const int f = (i < n && fabsf(h_error(H, pairs[i])) < threshold) ? 1 : 0;
        const unsigned bal = __ballot_sync(kFull, f);
        const int lane = t & 31, w = t >> 5;
        if (lane == 0) wsum[w] = __popc(bal);
        __syncthreads();
        int off = base_s;
        for (int k = 0; k < w; k++) off += wsum[k];
        if (f) inliers[off + __popc(bal & ((1u << lane) - 1u))] = i;
        __syncthreads();
        if (t == 0) {
            int s = 0;
            for (int k = 0; k < kFinalThreads / 32; k++) s += wsum[k];
            base_s += s;
        }
        __syncthreads();
    }
    const int m = base_s;
    if (t == 0) {
        *n_inliers = m;
        *loss_out = float(losses[best_s]);
    }
    auto comp = [](const float4& p, int c) { return c == 0 ? p.z : c == 1 ? p.w : c == 2 ? p.x : p.y; };
    bool refit = false;
    if (m >= 4) {
        // centroids, then mean absolute deviations: sequential sums over the
        // inliers in index order
        for (int pass = 0; pass < 2; pass++) {
            double acc = 0.0;
            for (int c0 = 0; c0 < m; c0 += kStage) {
                const int cnt = min(kStage, m - c0);
                __syncthreads();
                for (int i = t; i < cnt; i += kFinalThreads) stage[i] = pairs[inliers[c0 + i]];
                __syncthreads();
                if (t < 4) {
                    if (pass == 0)
                        for (int i = 0; i < cnt; i++) acc = dadd(acc, double(comp(stage[i], t)));
                    else
                        for (int i = 0; i < cnt; i++) acc = dadd(acc, fabs(dsub(double(comp(stage[i], t)), S.cen[t])));
                }
            }
            if (t < 4) {
                if (pass == 0) S.cen[t] = ddiv(acc, double(m));
                else S.mad[t] = ddiv(acc, double(m));
            }
            __syncthreads();
        }
        const double eps = DBL_EPSILON;
        const bool degenerate =
            fabs(S.mad[0]) < eps || fabs(S.mad[1]) < eps || fabs(S.mad[2]) < eps || fabs(S.mad[3]) < eps;
        if (!degenerate) {
            double acc = 0.0;
            int j = 0, k = 0;
            if (t < 45) tri_index(t, j, k);
            for (int c0 = 0; c0 < m; c0 += kStage) {
                const int cnt = min(kStage, m - c0);
                __syncthreads();
                for (int i = t; i < cnt; i += kFinalThreads) {
                    const float4 p = pairs[inliers[c0 + i]];
                    nstage[i] = make_double4(ddiv(dsub(double(p.x), S.cen[2]), S.mad[2]),
                                             ddiv(dsub(double(p.y), S.cen[3]), S.mad[3]),
                                             ddiv(dsub(double(p.z), S.cen[0]), S.mad[0]),
                                             ddiv(dsub(double(p.w), S.cen[1]), S.mad[1]));
                }
                __syncthreads();
                if (t < 45)
                    for (int q = 0; q < cnt; q++) {
                        const double4 v = nstage[q];
                        const double xj = lx_entry(j, v.x, v.y, v.z), xk = lx_entry(k, v.x, v.y, v.z);
                        const double yj = ly_entry(j, v.x, v.y, v.w), yk = ly_entry(k, v.x, v.y, v.w);
                        acc = dadd(acc, dadd(dmul(xj, xk), dmul(yj, yk)));
                    }
            }
            if (t < 45) {
                L[j * 9 + k] = acc;
                L[k * 9 + j] = acc;  // completeSymm
            }
            __syncthreads();
            if (t < 32) {
                for (int i = t; i < 81; i += 32) S.a[i] = L[i];
                __syncwarp();
                ls_finish_warp(S, Hf);
            }
            refit = true;
            __syncthreads();
        }
    }
    if (t < 9) Hout[t] = refit ? Hf[t] : H[t];
}

// ------------------------------------------------------------ raw channels
struct ChanArgs {
    const uint16_t* raw;
    size_t stride;  // elements
    int ow, oh;
    int ox[4], oy[4];
    float* out[4];
    int out_pitch[4];  // floats
    uint32_t mask;
    const float* lut;
};

// RawChannels (pyramidFusion.cpp:132-139) through a 65536-entry tone-curve
// table built on the host with the reference's expression.
__global__ void k_raw_channels(ChanArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.ow || y >= a.oh) return;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (!(a.mask & (1u << c))) continue;
        const uint16_t v = __ldg(a.raw + size_t(2 * y + a.oy[c]) * a.stride + 2 * x + a.ox[c]);
        a.out[c][size_t(y) * a.out_pitch[c] + x] = __ldg(a.lut + v);
    }
}

// ------------------------------------------------------------ integral
constexpr int IT = 32;  // integral tile edge

// Column pass (integral_sum_cols_image, SURF.metal:315-338): a running sum
// of (v - 0.5) down each column, sequential in float; written transposed
// (T[x][y]) through a shared-memory tile. The next tile is loaded into
// registers while one warp scans the current one.
__global__ void __launch_bounds__(256) k_integral_cols(const float* __restrict__ img, int pitch, int W, int H,
                                                       float* __restrict__ T, int tpitch) {
    __shared__ float tile[IT][IT + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x0 = blockIdx.x * IT;
    float nxt[IT / 8];
    auto load = [&](int y0) {
#pragma unroll
        for (int k = 0; k < IT / 8; k++) {
            const int r = ty + 8 * k, x = x0 + tx, y = y0 + r;
            nxt[k] = (x < W && y < H) ? __ldg(img + size_t(y) * pitch + x) : 0.0f;
        }
    };
    load(0);
    float acc = 0.0f;
    for (int y0 = 0; y0 < H; y0 += IT) {
#pragma unroll
        for (int k = 0; k < IT / 8; k++) tile[ty + 8 * k][tx] = nxt[k];
        __syncthreads();
        if (y0 + IT < H) load(y0 + IT);
        if (ty == 0) {
            const int rows = min(IT, H - y0);
#pragma unroll 8
            for (int r = 0; r < rows; r++) {
                acc = fadd(acc, fsub(tile[r][tx], 0.5f));
                tile[r][tx] = acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IT / 8; k++) {
            const int c = ty + 8 * k, x = x0 + c, y = y0 + tx;
            if (x < W && y < H) T[size_t(x) * tpitch + y] = tile[tx][c];
        }
        __syncthreads();
    }
}

// Row pass (integral_sum_rows_image, SURF.metal:340-421): a running sum of
// the column sums along each row, sequential in float, into the
// (W+1) x (H+1) sum image with a zero first row and column.
__global__ void __launch_bounds__(256) k_integral_rows(const float* __restrict__ T, int tpitch, int W, int H,
                                                       float* __restrict__ S, int spitch) {
    __shared__ float tile[IT][IT + 1];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int y0 = blockIdx.x * IT;
    float nxt[IT / 8];
    auto load = [&](int x0) {
#pragma unroll
        for (int k = 0; k < IT / 8; k++) {
            const int c = ty + 8 * k, x = x0 + c, y = y0 + tx;
            nxt[k] = (x < W && y < H) ? __ldg(T + size_t(x) * tpitch + y) : 0.0f;
        }
    };
    if (blockIdx.x == 0)
        for (int x = ty * IT + tx; x <= W; x += 8 * IT) S[x] = 0.0f;
    for (int k = 0; k < IT / 8; k++) {
        const int y = y0 + ty + 8 * k;
        if (tx == 0 && y < H) S[size_t(y + 1) * spitch] = 0.0f;
    }
    load(0);
    float acc = 0.0f;
    for (int x0 = 0; x0 < W; x0 += IT) {
#pragma unroll
        for (int k = 0; k < IT / 8; k++) tile[ty + 8 * k][tx] = nxt[k];
        __syncthreads();
        if (x0 + IT < W) load(x0 + IT);
        if (ty == 0) {
            const int cols = min(IT, W - x0);
#pragma unroll 8
            for (int c = 0; c < cols; c++) {
                acc = fadd(acc, tile[c][tx]);
                tile[c][tx] = acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < IT / 8; k++) {
            const int r = ty + 8 * k, y = y0 + r, x = x0 + tx;
            if (x < W && y < H) S[size_t(y + 1) * spitch + x + 1] = tile[tx][r];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ warps
struct WarpArgs {
    const float* fused;
    int fused_pitch;  // floats
    const void* input;
    int in_pitch;  // elements
    int iw, ih;
    float* out;
    int out_pitch;
    int w, h;
    float H[9];
    int count;  // 0: registerImage
};

template <class S>
__device__ __forceinline__ float4 rd4(const S* p) {
    if constexpr (std::is_same<S, float>::value) {
        return __ldg(reinterpret_cast<const float4*>(p));
    } else {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
}

__device__ __forceinline__ float lerp_(float a, float b, float t) { return fadd(a, fmul(t, fsub(b, a))); }

// registerAndFuse / registerImage (SURF.metal:489-538): pull-warp by H with
// exact bilinear sampling, clamp-to-edge, and the running mean.
template <class S>
__global__ void __launch_bounds__(256) k_register(WarpArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.w || y >= a.h) return;
    const float fx = float(x), fy = float(y);
    const float u = fadd(fadd(fmul(a.H[0], fx), fmul(a.H[1], fy)), a.H[2]);
    const float v = fadd(fadd(fmul(a.H[3], fx), fmul(a.H[4], fy)), a.H[5]);
    const float ww = fadd(fadd(fmul(a.H[6], fx), fmul(a.H[7], fy)), a.H[8]);
    const float xx = fminf(fmaxf(fdiv(u, ww), -1.0f), float(a.iw));
    const float yy = fminf(fmaxf(fdiv(v, ww), -1.0f), float(a.ih));
    const float x0f = floorf(xx), y0f = floorf(yy);
    const float ax = fsub(xx, x0f), ay = fsub(yy, y0f);
    const int x0 = int(x0f), y0 = int(y0f);
    const int xa = min(max(x0, 0), a.iw - 1), xb = min(max(x0 + 1, 0), a.iw - 1);
    const int ya = min(max(y0, 0), a.ih - 1), yb = min(max(y0 + 1, 0), a.ih - 1);
    const S* in = reinterpret_cast<const S*>(a.input);
    const float4 p00 = rd4(in + size_t(ya) * a.in_pitch + 4 * xa), p10 = rd4(in + size_t(ya) * a.in_pitch + 4 * xb);
    const float4 p01 = rd4(in + size_t(yb) * a.in_pitch + 4 * xa), p11 = rd4(in + size_t(yb) * a.in_pitch + 4 * xb);
    float4 s;
    {
        const float t = lerp_(p00.x, p10.x, ax), b = lerp_(p01.x, p11.x, ax);
        s.x = lerp_(t, b, ay);
    }
    {
        const float t = lerp_(p00.y, p10.y, ax), b = lerp_(p01.y, p11.y, ax);
        s.y = lerp_(t, b, ay);
    }
    {
        const float t = lerp_(p00.z, p10.z, ax), b = lerp_(p01.z, p11.z, ax);
        s.z = lerp_(t, b, ay);
    }
    {
        const float t = lerp_(p00.w, p10.w, ax), b = lerp_(p01.w, p11.w, ax);
        s.w = lerp_(t, b, ay);
    }
    float4* o = reinterpret_cast<float4*>(a.out + size_t(y) * a.out_pitch + 4 * x);
    if (a.count > 0) {
        const float4 f = *reinterpret_cast<const float4*>(a.fused + size_t(y) * a.fused_pitch + 4 * x);
        const float cm1 = float(a.count - 1), cn = float(a.count);
        s = make_float4(fdiv(fadd(fmul(cm1, f.x), s.x), cn), fdiv(fadd(fmul(cm1, f.y), s.y), cn),
                        fdiv(fadd(fmul(cm1, f.z), s.z), cn), fdiv(fadd(fmul(cm1, f.w), s.w), cn));
    }
    *o = s;
}

}  // namespace gls

namespace gls {
struct FusionScratch;
FusionScratch* fusion_scratch_new();
void fusion_scratch_delete(FusionScratch* f);
gls_status fuse_pyramid_impl(FusionScratch* F, const gls_image_view* frames, int n, const float* H, int levels,
                             float robustness, gls_image_view* out, cudaStream_t s);
}  // namespace gls

// ============================================================ host object
using namespace gls;

struct SurfSlotState {
    DevBuf kps, desc, count;
    int count_host = -1;  // -1: not read back since the last detection
    bool valid = false;
};

struct gls_surf {
    int device = 0, W = 0, H = 0, max_features = 1500, n_oct = 4, n_layers = 2;
    float threshold = 0.02f;
    int capacity = 1500;  // keypoints kept per slot
    DevBuf img, sum, colT, cand, cand_count, tables;
    SurfSlotState slot[GLS_SURF_SLOTS];
    DevBuf matches, matches_sorted, pairs;  // [jobs][pair_cap]
    int pair_cap = 0;
    int match_query = -1, match_train = -1;  // the slots of the last single match (job 0)
    std::map<std::pair<int, int>, DevBuf> sample_tables;
    DevBuf models, losses, inliers, n_inliers, Hdev, loss;
    DevBuf raw, lut;
    float lut_black = NAN, lut_white = NAN, lut_exp = NAN;
    std::vector<float> lut_host;
    FusionScratch* fusion = nullptr;
    uint64_t launches = 0;
};

namespace {

gls_status check_surf(gls_surf* s) {
    if (!s) return set_error(GLS_ERR_INVALID_ARG, "NULL detector");
    GLS_CUDA(cudaSetDevice(s->device));
    return GLS_OK;
}

gls_status launch_check(gls_surf* s, const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
    s->launches++;
    return GLS_OK;
}

// getGaussianKernel (SURF.cpp:394-425) for sigma > 0
std::vector<float> gaussian_kernel(int n, float sigma) {
    const float scale2X = float(-0.5 / double(sigma * sigma));
    float sum = 0;
    std::vector<float> k(n);
    for (int i = 0; i < n; i++) {
        const float x = float(i - (n - 1) * 0.5);
        k[i] = std::exp(scale2X * x * x);
        sum += k[i];
    }
    sum = float(1. / sum);
    for (auto& v : k) v *= sum;
    return k;
}

DescTables make_tables() {
    DescTables t{};
    const auto g = gaussian_kernel(13, 2.5f);
    for (int i = -6; i <= 6; i++)
        for (int j = -6; j <= 6; j++)
            if (i * i + j * j <= 36) {
                t.apt_x[t.n_ori] = float(i);
                t.apt_y[t.n_ori] = float(j);
                t.aptw[t.n_ori++] = g[i + 6] * g[j + 6];
            }
    const auto gd = gaussian_kernel(20, 3.3f);
    for (int i = 0; i < 20; i++)
        for (int j = 0; j < 20; j++) t.dw[i * 20 + j] = gd[i] * gd[j];
    return t;
}

// toneCurve / sigmoid (pyramidFusion.cpp:92-104) in the reference's mix of
// float and double.
float sigmoid(float x, float s) { return float(0.5 * (std::tanh(double(s * x) - 0.3 * s) + 1)); }
float tone_curve(float x, float s) {
    const float p = float(std::pow(0.95 * x, 0.5));
    return (sigmoid(p, s) - sigmoid(0.0f, s)) / (sigmoid(1.0f, s) - sigmoid(0.0f, s));
}

// mt19937 (default seed) with a mask-and-reject uniform integer in [0, n-1]:
// the 4-index sets of RTL::RANSAC::GenerateModel (RTL/RANSAC.hpp:95-99), each
// in ascending order.
std::vector<int> ransac_samples(int iterations, int n) {
    std::mt19937 g;
    const uint32_t range = uint32_t(n);
    int w = 0;
    while (w < 32 && (uint64_t(1) << w) < range) w++;
    const uint32_t mask = w >= 32 ? 0xffffffffu : ((1u << w) - 1u);
    std::vector<int> out(size_t(iterations) * 4);
    for (int it = 0; it < iterations; it++) {
        std::set<int> s;
        while (s.size() < 4) {
            int v = 0;
            if (range > 1) {
                uint32_t u;
                do {
                    u = uint32_t(g()) & mask;
                } while (u >= range);
                v = int(u);
            }
            s.insert(v);
            if (range < 4 && s.size() == range) break;
        }
        int k = 0;
        for (int v : s) out[size_t(it) * 4 + k++] = v;
        for (; k < 4; k++) out[size_t(it) * 4 + k] = *s.begin();
    }
    return out;
}

// the RANSAC sample table for n pairs (cached per (n, iterations))
gls_status sample_table(gls_surf* s, int n, int iters, const int** out, cudaStream_t st) {
    auto key = std::make_pair(n, iters);
    auto it = s->sample_tables.find(key);
    if (it == s->sample_tables.end()) {
        const std::vector<int> smp = ransac_samples(iters, n);
        DevBuf b;
        GLS_TRY(b.ensure(smp.size() * sizeof(int)));
        GLS_CUDA(cudaMemcpyAsync(b.p, smp.data(), smp.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        GLS_CUDA(cudaStreamSynchronize(st));
        it = s->sample_tables.emplace(key, b).first;
    }
    *out = reinterpret_cast<const int*>(it->second.p);
    return GLS_OK;
}

// RANSAC + refit for jobs 0..J-1 whose pairs are in s->pairs (cap per job)
// and whose pair counts are ns[j]; leaves H [J][9], inliers, counts on the
// device.
gls_status run_ransac(gls_surf* s, const std::vector<int>& ns, float threshold, int iters, cudaStream_t st) {
    const int J = int(ns.size());
    const size_t cap = size_t(std::max(s->pair_cap, 1));
    RansacJobs rj{};
    for (int j = 0; j < J; j++) {
        if (ns[j] < 4) return set_error(GLS_ERR_DEGENERATE, "RANSAC needs at least 4 point pairs, got %d", ns[j]);
        rj.j[j].pairs = reinterpret_cast<const float4*>(s->pairs.p) + size_t(j) * cap;
        rj.j[j].n = ns[j];
        GLS_TRY(sample_table(s, ns[j], iters, &rj.j[j].samples, st));
    }
    GLS_TRY(s->models.ensure(size_t(J) * iters * 9 * sizeof(float)));
    GLS_TRY(s->losses.ensure(size_t(J) * iters * sizeof(int)));
    GLS_TRY(s->inliers.ensure(size_t(J) * cap * sizeof(int)));
    GLS_TRY(s->n_inliers.ensure(size_t(J) * sizeof(int)));
    GLS_TRY(s->Hdev.ensure(size_t(J) * 9 * sizeof(float)));
    GLS_TRY(s->loss.ensure(size_t(J) * sizeof(float)));
    k_ransac_models<<<dim3((iters + kHypWarps - 1) / kHypWarps, J), 32 * kHypWarps, 0, st>>>(
        rj, iters, threshold, reinterpret_cast<float*>(s->models.p), reinterpret_cast<int*>(s->losses.p));
    GLS_TRY(launch_check(s, "k_ransac_models"));
    k_ransac_final<<<J, kFinalThreads, 0, st>>>(rj, int(cap), reinterpret_cast<const float*>(s->models.p),
                                                reinterpret_cast<const int*>(s->losses.p), iters, threshold,
                                                reinterpret_cast<int*>(s->inliers.p),
                                                reinterpret_cast<int*>(s->n_inliers.p),
                                                reinterpret_cast<float*>(s->Hdev.p), reinterpret_cast<float*>(s->loss.p));
    GLS_TRY(launch_check(s, "k_ransac_final"));
    return GLS_OK;
}

// copies job 0's homography and inliers to the host (synchronising)
gls_status ransac_result(gls_surf* s, float* H, int32_t* inliers, int32_t* n_inl, cudaStream_t st) {
    int ni = 0;
    GLS_CUDA(cudaMemcpyAsync(H, s->Hdev.p, 9 * sizeof(float), cudaMemcpyDeviceToHost, st));
    GLS_CUDA(cudaMemcpyAsync(&ni, s->n_inliers.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    GLS_CUDA(cudaStreamSynchronize(st));
    if (n_inl) *n_inl = ni;
    if (inliers && ni > 0)
        GLS_CUDA(cudaMemcpy(inliers, s->inliers.p, size_t(ni) * sizeof(int), cudaMemcpyDeviceToHost));
    return GLS_OK;
}

gls_status ensure_pairs(gls_surf* s, int jobs, int cap) {
    s->pair_cap = std::max(s->pair_cap, cap);
    const size_t c = size_t(std::max(s->pair_cap, 1));
    GLS_TRY(s->matches.ensure(size_t(jobs) * c * sizeof(gls_match)));
    GLS_TRY(s->matches_sorted.ensure(size_t(jobs) * c * sizeof(gls_match)));
    GLS_TRY(s->pairs.ensure(size_t(jobs) * c * sizeof(float4)));
    return GLS_OK;
}

// match jobs (query slot, train slot) into matches / pairs job by job
gls_status run_match(gls_surf* s, const std::vector<std::pair<int, int>>& qt, cudaStream_t st) {
    const int J = int(qt.size());
    if (s->pair_cap != s->capacity) s->pair_cap = 0;
    GLS_TRY(ensure_pairs(s, J, s->capacity));
    MatchJobs mj{};
    for (int j = 0; j < J; j++) {
        const SurfSlotState &q = s->slot[qt[j].first], &t = s->slot[qt[j].second];
        mj.j[j] = {reinterpret_cast<const float*>(q.desc.p), reinterpret_cast<const int*>(q.count.p),
                   reinterpret_cast<const gls_keypoint*>(q.kps.p), reinterpret_cast<const float*>(t.desc.p),
                   reinterpret_cast<const int*>(t.count.p), reinterpret_cast<const gls_keypoint*>(t.kps.p)};
    }
    const int cap = s->pair_cap;
    const int warps = 4;
    k_match<<<dim3((s->capacity + warps - 1) / warps, J), 32 * warps, 0, st>>>(
        mj, cap, reinterpret_cast<gls_match*>(s->matches.p));
    GLS_TRY(launch_check(s, "k_match"));
    k_match_rank<<<dim3((s->capacity + 255) / 256, J), 256, 0, st>>>(
        mj, cap, reinterpret_cast<const gls_match*>(s->matches.p), reinterpret_cast<gls_match*>(s->matches_sorted.p),
        reinterpret_cast<float4*>(s->pairs.p));
    GLS_TRY(launch_check(s, "k_match_rank"));
    return GLS_OK;
}

}  // namespace

extern "C" {

gls_status gls_surf_create(int32_t device, int32_t width, int32_t height, int32_t max_features, int32_t n_octaves,
                           int32_t n_octave_layers, float hessian_threshold, gls_surf** out) {
    clear_error();
    if (!out) return set_error(GLS_ERR_INVALID_ARG, "NULL output");
    *out = nullptr;
    if (width < 1 || height < 1 || width > 32768 || height > 32768)
        return set_error(GLS_ERR_INVALID_ARG, "image size %dx%d out of range", width, height);
    if (n_octaves < 1 || n_octaves > kMaxOctaves)
        return set_error(GLS_ERR_INVALID_ARG, "n_octaves must be 1..%d", kMaxOctaves);
    if (n_octave_layers != 2)
        return set_error(GLS_ERR_UNSUPPORTED, "only 2 layers per octave (the reference's setting) are served");
    GLS_CUDA(cudaSetDevice(device));
    auto* s = new gls_surf();
    s->device = device;
    s->W = width;
    s->H = height;
    s->max_features = max_features;
    s->n_oct = n_octaves;
    s->n_layers = n_octave_layers;
    s->threshold = hessian_threshold;
    s->capacity = max_features < 0 ? kMaxKeypoints : std::min(max_features, kMaxKeypoints);
    auto fail = [&](gls_status st) {
        gls_surf_destroy(s);
        return st;
    };
    const size_t n = size_t(width) * height;
    gls_status st;
    if ((st = s->img.ensure(n * sizeof(float))) != GLS_OK) return fail(st);
    if ((st = s->sum.ensure(size_t(width + 1) * (height + 1) * sizeof(float))) != GLS_OK) return fail(st);
    if ((st = s->colT.ensure(n * sizeof(float))) != GLS_OK) return fail(st);
    if ((st = s->cand.ensure(size_t(kMaxKeypoints) * sizeof(gls_keypoint))) != GLS_OK) return fail(st);
    if ((st = s->cand_count.ensure(sizeof(int))) != GLS_OK) return fail(st);
    if ((st = s->tables.ensure(sizeof(DescTables))) != GLS_OK) return fail(st);
    const DescTables t = make_tables();
    if (cudaMemcpy(s->tables.p, &t, sizeof(t), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(set_error(GLS_ERR_CUDA, "upload of the descriptor tables failed"));
    for (auto& sl : s->slot) {
        if ((st = sl.kps.ensure(size_t(std::max(s->capacity, 1)) * sizeof(gls_keypoint))) != GLS_OK) return fail(st);
        if ((st = sl.desc.ensure(size_t(std::max(s->capacity, 1)) * 64 * sizeof(float))) != GLS_OK) return fail(st);
        if ((st = sl.count.ensure(sizeof(int))) != GLS_OK) return fail(st);
        if (cudaMemset(sl.count.p, 0, sizeof(int)) != cudaSuccess)
            return fail(set_error(GLS_ERR_CUDA, "cudaMemset failed"));
    }
    *out = s;
    return GLS_OK;
}

gls_status gls_surf_destroy(gls_surf* s) {
    if (!s) return GLS_OK;
    cudaSetDevice(s->device);
    for (DevBuf* b : {&s->img, &s->sum, &s->colT, &s->cand, &s->cand_count, &s->tables, &s->matches,
                      &s->matches_sorted, &s->pairs, &s->models, &s->losses, &s->inliers, &s->n_inliers, &s->Hdev,
                      &s->loss, &s->raw, &s->lut})
        b->release();
    for (auto& kv : s->sample_tables) kv.second.release();
    if (s->fusion) fusion_scratch_delete(s->fusion);
    for (auto& sl : s->slot) {
        sl.kps.release();
        sl.desc.release();
        sl.count.release();
    }
    delete s;
    return GLS_OK;
}

gls_status gls_surf_detect_and_compute(gls_surf* s, const gls_image_view* img, int32_t slot, uint32_t flags,
                                       void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (!img || !img->data) return set_error(GLS_ERR_INVALID_ARG, "NULL image");
    if (slot < 0 || slot >= GLS_SURF_SLOTS) return set_error(GLS_ERR_INVALID_ARG, "slot %d out of range", slot);
    if (img->channels != 1 || img->dtype != GLS_F32)
        return set_error(GLS_ERR_INVALID_ARG, "image must be single-channel GLS_F32");
    if (img->width != s->W || img->height != s->H)
        return set_error(GLS_ERR_INVALID_ARG, "image is %dx%d, detector serves %dx%d", img->width, img->height, s->W,
                         s->H);
    const size_t stride = img->stride_bytes ? img->stride_bytes : size_t(img->width) * 4;
    if (stride % 4 || stride < size_t(img->width) * 4) return set_error(GLS_ERR_INVALID_ARG, "bad image stride");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const float* src = reinterpret_cast<const float*>(img->data);
    int pitch = int(stride / 4);
    if (flags & GLS_HOST_IO) {
        GLS_CUDA(cudaMemcpy2DAsync(s->img.p, size_t(s->W) * 4, img->data, stride, size_t(s->W) * 4, s->H,
                                   cudaMemcpyHostToDevice, st));
        src = reinterpret_cast<const float*>(s->img.p);
        pitch = s->W;
    }
    const int W = s->W, H = s->H;
    const int tpitch = H;
    float* T = reinterpret_cast<float*>(s->colT.p);
    float* S = reinterpret_cast<float*>(s->sum.p);
    k_integral_cols<<<(W + IT - 1) / IT, dim3(32, 8), 0, st>>>(src, pitch, W, H, T, tpitch);
    GLS_TRY(launch_check(s, "k_integral_cols"));
    k_integral_rows<<<(H + IT - 1) / IT, dim3(32, 8), 0, st>>>(T, tpitch, W, H, S, W + 1);
    GLS_TRY(launch_check(s, "k_integral_rows"));
    // fastHessianDetector (SURF.cpp:1229-1286)
    DetectArgs da{};
    da.n_oct = s->n_oct;
    da.sum = S;
    da.sum_pitch = W + 1;
    da.threshold = s->threshold;
    da.per_axis = (flags & GLS_SURF_CORRECTED) ? 1 : 0;
    da.cand = reinterpret_cast<gls_keypoint*>(s->cand.p);
    da.cand_count = reinterpret_cast<int*>(s->cand_count.p);
    int blocks = 0;
    for (int o = 0; o < s->n_oct; o++) {
        OctaveDev& O = da.oct[o];
        O.step = 1 << o;
        for (int l = 0; l < kLayers; l++) O.layer[l] = make_layer(W + 1, H + 1, (9 + 6 * l) << o, O.step);
        O.lw = W / O.step;
        O.lh = H / O.step;
        O.tiles_x = std::max(1, (O.lw + DT_X - 1) / DT_X);
        O.tiles_y = std::max(1, (O.lh + DT_Y - 1) / DT_Y);
        O.block0 = blocks;
        blocks += O.tiles_x * O.tiles_y;
    }
    GLS_CUDA(cudaMemsetAsync(s->cand_count.p, 0, sizeof(int), st));
    k_hessian_nms<<<blocks, 256, 0, st>>>(da);
    GLS_TRY(launch_check(s, "k_hessian_nms"));
    SurfSlotState& sl = s->slot[slot];
    const int keep = s->capacity;
    k_keypoint_rank<<<(kMaxKeypoints + 255) / 256, 256, 0, st>>>(
        reinterpret_cast<const gls_keypoint*>(s->cand.p), reinterpret_cast<const int*>(s->cand_count.p), keep,
        reinterpret_cast<gls_keypoint*>(sl.kps.p), reinterpret_cast<int*>(sl.count.p));
    GLS_TRY(launch_check(s, "k_keypoint_rank"));
    DescArgs ga{};
    ga.img = src;
    ga.img_pitch = pitch;
    ga.iw = W;
    ga.ih = H;
    ga.sum = S;
    ga.sum_pitch = W + 1;
    ga.sw = W + 1;
    ga.sh = H + 1;
    ga.tab = reinterpret_cast<const DescTables*>(s->tables.p);
    ga.kps = reinterpret_cast<gls_keypoint*>(sl.kps.p);
    ga.count = reinterpret_cast<const int*>(sl.count.p);
    ga.desc = reinterpret_cast<float*>(sl.desc.p);
    ga.all = (flags & GLS_SURF_CORRECTED) ? 1 : 0;
    if (keep > 0) {
        k_describe<<<keep, kDescThreads, 0, st>>>(ga);
        GLS_TRY(launch_check(s, "k_describe"));
    }
    sl.count_host = -1;
    sl.valid = true;
    if (s->match_query == slot || s->match_train == slot) s->match_query = s->match_train = -1;
    if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(st));
    return GLS_OK;
}

static gls_status slot_count(gls_surf* s, int slot, cudaStream_t st, int* n) {
    SurfSlotState& sl = s->slot[slot];
    if (!sl.valid) return set_error(GLS_ERR_INVALID_ARG, "slot %d holds no detection", slot);
    if (sl.count_host < 0) {
        int c = 0;
        GLS_CUDA(cudaMemcpyAsync(&c, sl.count.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        GLS_CUDA(cudaStreamSynchronize(st));
        sl.count_host = c;
    }
    *n = sl.count_host;
    return GLS_OK;
}

gls_status gls_surf_features(gls_surf* s, int32_t slot, gls_keypoint* kps, float* desc, int32_t capacity, int32_t* n,
                             void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (slot < 0 || slot >= GLS_SURF_SLOTS) return set_error(GLS_ERR_INVALID_ARG, "slot %d out of range", slot);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int c = 0;
    GLS_TRY(slot_count(s, slot, st, &c));
    if (n) *n = c;
    const int m = std::min(c, std::max(capacity, 0));
    if (kps && m > 0)
        GLS_CUDA(cudaMemcpyAsync(kps, s->slot[slot].kps.p, size_t(m) * sizeof(gls_keypoint), cudaMemcpyDeviceToHost, st));
    if (desc && m > 0)
        GLS_CUDA(cudaMemcpyAsync(desc, s->slot[slot].desc.p, size_t(m) * 64 * sizeof(float), cudaMemcpyDeviceToHost,
                                 st));
    GLS_CUDA(cudaStreamSynchronize(st));
    return GLS_OK;
}

gls_status gls_surf_load_features(gls_surf* s, int32_t slot, const gls_keypoint* kps, const float* desc, int32_t n,
                                  uint32_t flags, void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (slot < 0 || slot >= GLS_SURF_SLOTS) return set_error(GLS_ERR_INVALID_ARG, "slot %d out of range", slot);
    if (n < 0 || n > s->capacity)
        return set_error(GLS_ERR_INVALID_ARG, "%d features, the detector keeps at most %d", n, s->capacity);
    if (n > 0 && (!kps || !desc)) return set_error(GLS_ERR_INVALID_ARG, "NULL features");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const cudaMemcpyKind kind = (flags & GLS_HOST_IO) ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    SurfSlotState& sl = s->slot[slot];
    if (n > 0) {
        GLS_CUDA(cudaMemcpyAsync(sl.kps.p, kps, size_t(n) * sizeof(gls_keypoint), kind, st));
        GLS_CUDA(cudaMemcpyAsync(sl.desc.p, desc, size_t(n) * 64 * sizeof(float), kind, st));
    }
    // the count is written by a kernel on the stream (no host buffer has to
    // outlive the call, and the write can be recorded in a graph)
    k_store_count<<<1, 1, 0, st>>>(static_cast<int*>(sl.count.p), n);
    GLS_TRY(launch_check(s, "store_count"));
    if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(st));
    sl.count_host = n;
    sl.valid = true;
    if (s->match_query == slot || s->match_train == slot) s->match_query = s->match_train = -1;
    return GLS_OK;
}

gls_status gls_surf_plane(gls_surf* s, int32_t which, gls_image_view* view) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (!view) return set_error(GLS_ERR_INVALID_ARG, "NULL view");
    if (which != GLS_SURF_PLANE_INTEGRAL) return set_error(GLS_ERR_INVALID_ARG, "unknown plane %d", which);
    *view = gls_image_view{s->sum.p, s->W + 1, s->H + 1, 1, GLS_F32, size_t(s->W + 1) * sizeof(float)};
    return GLS_OK;
}

gls_status gls_surf_match(gls_surf* s, int32_t query_slot, int32_t train_slot, gls_match* matches, int32_t capacity,
                          int32_t* n, void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (query_slot < 0 || query_slot >= GLS_SURF_SLOTS || train_slot < 0 || train_slot >= GLS_SURF_SLOTS)
        return set_error(GLS_ERR_INVALID_ARG, "slot out of range");
    if (!s->slot[query_slot].valid || !s->slot[train_slot].valid)
        return set_error(GLS_ERR_INVALID_ARG, "slot holds no detection");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GLS_TRY(run_match(s, {{query_slot, train_slot}}, st));
    s->match_query = query_slot;
    s->match_train = train_slot;
    if (matches || n) {
        int c = 0;
        GLS_TRY(slot_count(s, query_slot, st, &c));
        if (n) *n = c;
        const int m = std::min(c, std::max(capacity, 0));
        if (matches && m > 0)
            GLS_CUDA(cudaMemcpyAsync(matches, s->matches_sorted.p, size_t(m) * sizeof(gls_match),
                                     cudaMemcpyDeviceToHost, st));
        GLS_CUDA(cudaStreamSynchronize(st));
    }
    return GLS_OK;
}

gls_status gls_surf_find_homography(gls_surf* s, float threshold, int32_t max_iterations, float* H, int32_t* inliers,
                                    int32_t* n_inliers, void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (!H) return set_error(GLS_ERR_INVALID_ARG, "NULL H");
    if (max_iterations < 1) return set_error(GLS_ERR_INVALID_ARG, "max_iterations must be positive");
    if (s->match_query < 0) return set_error(GLS_ERR_INVALID_ARG, "no match result (call gls_surf_match first)");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int n = 0;
    GLS_TRY(slot_count(s, s->match_query, st, &n));
    GLS_TRY(run_ransac(s, {n}, threshold, max_iterations, st));
    return ransac_result(s, H, inliers, n_inliers, st);
}

gls_status gls_find_homography(gls_surf* ctx, const float* pairs, int32_t n, float threshold, int32_t max_iterations,
                               float* H, int32_t* inliers, int32_t* n_inliers, void* stream) {
    clear_error();
    GLS_TRY(check_surf(ctx));
    if (!pairs || !H) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (max_iterations < 1) return set_error(GLS_ERR_INVALID_ARG, "max_iterations must be positive");
    if (n < 4) return set_error(GLS_ERR_DEGENERATE, "RANSAC needs at least 4 point pairs, got %d", n);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    GLS_TRY(ensure_pairs(ctx, 1, n));
    GLS_CUDA(cudaMemcpyAsync(ctx->pairs.p, pairs, size_t(n) * sizeof(float4), cudaMemcpyHostToDevice, st));
    ctx->match_query = ctx->match_train = -1;  // the pair buffer now holds host pairs
    GLS_TRY(run_ransac(ctx, {n}, threshold, max_iterations, st));
    return ransac_result(ctx, H, inliers, n_inliers, st);
}

gls_status gls_surf_register_frames(gls_surf* s, const int32_t* ref_slots, int32_t n_channels,
                                    const int32_t* frame_slots, int32_t n_frames, float threshold,
                                    int32_t max_iterations, int32_t scale_to_full, float* H, void* stream) {
    clear_error();
    GLS_TRY(check_surf(s));
    if (!ref_slots || !frame_slots || !H) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (n_channels < 1 || n_frames < 1 || n_channels * n_frames > kMaxJobs)
        return set_error(GLS_ERR_INVALID_ARG, "n_channels x n_frames must be 1..%d", kMaxJobs);
    if (max_iterations < 1) return set_error(GLS_ERR_INVALID_ARG, "max_iterations must be positive");
    auto ok = [&](int sl) { return sl >= 0 && sl < GLS_SURF_SLOTS && s->slot[sl].valid; };
    for (int c = 0; c < n_channels; c++)
        if (!ok(ref_slots[c])) return set_error(GLS_ERR_INVALID_ARG, "reference slot %d holds no detection", ref_slots[c]);
    for (int i = 0; i < n_channels * n_frames; i++)
        if (!ok(frame_slots[i])) return set_error(GLS_ERR_INVALID_ARG, "frame slot %d holds no detection", frame_slots[i]);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    std::vector<std::pair<int, int>> qt;
    std::vector<int> ns;
    for (int f = 0; f < n_frames; f++)
        for (int c = 0; c < n_channels; c++) {
            qt.push_back({ref_slots[c], frame_slots[f * n_channels + c]});
            int n = 0;
            GLS_TRY(slot_count(s, ref_slots[c], st, &n));
            ns.push_back(n);
        }
    GLS_TRY(run_match(s, qt, st));
    s->match_query = s->match_train = -1;
    GLS_TRY(run_ransac(s, ns, threshold, max_iterations, st));
    std::vector<float> Hj(qt.size() * 9);
    GLS_CUDA(cudaMemcpyAsync(Hj.data(), s->Hdev.p, Hj.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    GLS_CUDA(cudaStreamSynchronize(st));
    for (int f = 0; f < n_frames; f++) {
        float acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < n_channels; c++)  // running average, pyramidFusion.cpp:338-339
            for (int i = 0; i < 9; i++)
                acc[i] = (Hj[size_t(f * n_channels + c) * 9 + i] + acc[i] * float(c)) / float(c + 1);
        if (scale_to_full) GLS_TRY(gls_scale_homography(acc, 2.0f, acc));
        std::memcpy(H + size_t(f) * 9, acc, sizeof(acc));
    }
    return GLS_OK;
}

gls_status gls_scale_homography(const float* H, float scale, float* out) {
    (void)scale;  // Homography.hpp:30-34 ignores it
    if (!H || !out) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    const float h[9] = {H[0], H[1], H[2] * 2.0f, H[3], H[4], H[5] * 2.0f, H[6] * 0.5f, H[7] * 0.5f, H[8]};
    std::memcpy(out, h, sizeof(h));
    return GLS_OK;
}

gls_status gls_raw_channels(gls_surf* ctx, const uint16_t* raw, int32_t width, int32_t height, size_t stride_bytes,
                            int32_t bayer_pattern, float black_level, float white_level, float exposure_multiplier,
                            uint32_t channel_mask, gls_image_view* out, uint32_t flags, void* stream) {
    clear_error();
    GLS_TRY(check_surf(ctx));
    if (!raw || !out) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (bayer_pattern < 0 || bayer_pattern > 3) return set_error(GLS_ERR_INVALID_ARG, "bad Bayer pattern");
    if (width < 2 || height < 2) return set_error(GLS_ERR_INVALID_ARG, "raw image too small");
    if ((channel_mask & 0xfu) == 0 || (channel_mask & ~0xfu)) return set_error(GLS_ERR_INVALID_ARG, "bad channel mask");
    const size_t stride = stride_bytes ? stride_bytes : size_t(width) * 2;
    if (stride % 2 || stride < size_t(width) * 2) return set_error(GLS_ERR_INVALID_ARG, "bad raw stride");
    const int ow = width / 2, oh = height / 2;
    ChanArgs a{};
    static const int kHostBayer[4][4][2] = {{{1, 0}, {0, 0}, {0, 1}, {1, 1}},
                                            {{0, 1}, {0, 0}, {1, 0}, {1, 1}},
                                            {{0, 0}, {1, 0}, {1, 1}, {0, 1}},
                                            {{1, 1}, {1, 0}, {0, 0}, {0, 1}}};
    for (int c = 0; c < 4; c++) {
        a.ox[c] = kHostBayer[bayer_pattern][c][0];
        a.oy[c] = kHostBayer[bayer_pattern][c][1];
        if (!(channel_mask & (1u << c))) continue;
        const gls_image_view& v = out[c];
        if (!v.data || v.channels != 1 || v.dtype != GLS_F32 || v.width != ow || v.height != oh)
            return set_error(GLS_ERR_INVALID_ARG, "output %d must be a %dx%d single-channel GLS_F32 view", c, ow, oh);
        const size_t os = v.stride_bytes ? v.stride_bytes : size_t(ow) * 4;
        if (os % 4 || os < size_t(ow) * 4) return set_error(GLS_ERR_INVALID_ARG, "bad output stride");
        a.out[c] = reinterpret_cast<float*>(v.data);
        a.out_pitch[c] = int(os / 4);
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (!(ctx->lut_black == black_level && ctx->lut_white == white_level && ctx->lut_exp == exposure_multiplier)) {
        ctx->lut_host.resize(65536);
        for (int v = 0; v < 65536; v++) {
            const float x = exposure_multiplier * (float(v) - black_level) / white_level;
            ctx->lut_host[v] = tone_curve(std::clamp(x, 0.0f, 1.0f), 3.5f);
        }
        GLS_TRY(ctx->lut.ensure(65536 * sizeof(float)));
        GLS_CUDA(cudaMemcpyAsync(ctx->lut.p, ctx->lut_host.data(), 65536 * sizeof(float), cudaMemcpyHostToDevice, st));
        ctx->lut_black = black_level;
        ctx->lut_white = white_level;
        ctx->lut_exp = exposure_multiplier;
    }
    const uint16_t* src = raw;
    size_t spx = stride / 2;
    if (flags & GLS_HOST_IO) {
        GLS_TRY(ctx->raw.ensure(size_t(width) * height * 2));
        GLS_CUDA(cudaMemcpy2DAsync(ctx->raw.p, size_t(width) * 2, raw, stride, size_t(width) * 2, height,
                                   cudaMemcpyHostToDevice, st));
        src = reinterpret_cast<const uint16_t*>(ctx->raw.p);
        spx = width;
    }
    a.raw = src;
    a.stride = spx;
    a.ow = ow;
    a.oh = oh;
    a.mask = channel_mask;
    a.lut = reinterpret_cast<const float*>(ctx->lut.p);
    k_raw_channels<<<dim3((ow + 255) / 256, oh), 256, 0, st>>>(a);
    GLS_TRY(launch_check(ctx, "k_raw_channels"));
    if (flags & (GLS_SYNC | GLS_HOST_IO)) GLS_CUDA(cudaStreamSynchronize(st));
    return GLS_OK;
}

static gls_status warp(const gls_image_view* fused, const gls_image_view* input, gls_image_view* out, const float* H,
                       int count, void* stream) {
    if (!input || !out || !H || !input->data || !out->data) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (input->channels != 4 || (input->dtype != GLS_F32 && input->dtype != GLS_F16))
        return set_error(GLS_ERR_INVALID_ARG, "input must be RGBA GLS_F32 or GLS_F16");
    if (out->channels != 4 || out->dtype != GLS_F32) return set_error(GLS_ERR_INVALID_ARG, "out must be RGBA GLS_F32");
    if (input->width < 1 || input->height < 1 || out->width < 1 || out->height < 1)
        return set_error(GLS_ERR_INVALID_ARG, "empty image");
    const size_t ies = input->dtype == GLS_F32 ? 4 : 2;
    const size_t is = input->stride_bytes ? input->stride_bytes : size_t(input->width) * 4 * ies;
    const size_t os = out->stride_bytes ? out->stride_bytes : size_t(out->width) * 16;
    if (is % (4 * ies) || os % 16 || (reinterpret_cast<uintptr_t>(input->data) % (4 * ies)) ||
        (reinterpret_cast<uintptr_t>(out->data) % 16))
        return set_error(GLS_ERR_INVALID_ARG, "pixel rows must be aligned to whole RGBA pixels");
    WarpArgs a{};
    if (count > 0) {
        if (!fused || !fused->data || fused->channels != 4 || fused->dtype != GLS_F32 || fused->width != out->width ||
            fused->height != out->height)
            return set_error(GLS_ERR_INVALID_ARG, "fused must be RGBA GLS_F32 of the output's size");
        const size_t fs = fused->stride_bytes ? fused->stride_bytes : size_t(fused->width) * 16;
        if (fs % 16 || (reinterpret_cast<uintptr_t>(fused->data) % 16))
            return set_error(GLS_ERR_INVALID_ARG, "fused rows must be 16-byte aligned");
        a.fused = reinterpret_cast<const float*>(fused->data);
        a.fused_pitch = int(fs / 4);
    }
    a.input = input->data;
    a.in_pitch = int(is / ies);
    a.iw = input->width;
    a.ih = input->height;
    a.out = reinterpret_cast<float*>(out->data);
    a.out_pitch = int(os / 4);
    a.w = out->width;
    a.h = out->height;
    for (int i = 0; i < 9; i++) a.H[i] = H[i];
    a.count = count;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const dim3 grid((out->width + 255) / 256, out->height);
    if (input->dtype == GLS_F32) k_register<float><<<grid, 256, 0, st>>>(a);
    else k_register<__half><<<grid, 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "k_register launch: %s", cudaGetErrorString(e));
    return GLS_OK;
}

gls_status gls_register_and_fuse(const gls_image_view* fused, const gls_image_view* input, gls_image_view* out,
                                 const float* H, int32_t count, void* stream) {
    clear_error();
    if (count < 1) return set_error(GLS_ERR_INVALID_ARG, "count must be >= 1");
    return warp(fused, input, out, H, count, stream);
}

gls_status gls_fuse_pyramid(gls_surf* ctx, const gls_image_view* frames, int32_t n_frames, const float* H,
                            int32_t levels, float robustness, gls_image_view* out, void* stream) {
    clear_error();
    GLS_TRY(check_surf(ctx));
    if (!frames || !out || !out->data || (n_frames > 1 && !H)) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (n_frames < 1) return set_error(GLS_ERR_INVALID_ARG, "no frames");
    if (levels < 1 || levels > GLS_MAX_LEVELS) return set_error(GLS_ERR_INVALID_ARG, "levels must be 1..%d", GLS_MAX_LEVELS);
    if (!(robustness >= 0.f)) return set_error(GLS_ERR_INVALID_ARG, "robustness must be >= 0");
    const int W = frames[0].width, Hh = frames[0].height;
    if ((W >> (levels - 1)) < 1 || (Hh >> (levels - 1)) < 1) return set_error(GLS_ERR_INVALID_ARG, "too many levels");
    if (out->width != W || out->height != Hh || out->channels != 4 || (out->dtype != GLS_F32 && out->dtype != GLS_F16))
        return set_error(GLS_ERR_INVALID_ARG, "out must be a %dx%d RGBA GLS_F32 or GLS_F16 view", W, Hh);
    const size_t oes = out->dtype == GLS_F32 ? 4 : 2;
    if ((out->stride_bytes && out->stride_bytes % (4 * oes)) || (reinterpret_cast<uintptr_t>(out->data) % (4 * oes)))
        return set_error(GLS_ERR_INVALID_ARG, "out rows must be aligned to whole RGBA pixels");
    if (!ctx->fusion) ctx->fusion = fusion_scratch_new();
    return fuse_pyramid_impl(ctx->fusion, frames, n_frames, H, levels, robustness, out,
                             reinterpret_cast<cudaStream_t>(stream));
}

gls_status gls_register_image(const gls_image_view* input, gls_image_view* out, const float* H, void* stream) {
    clear_error();
    return warp(nullptr, input, out, H, 0, stream);
}

}  // extern "C"
