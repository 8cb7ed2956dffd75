// gls_common.cuh — device helpers shared by the raw-path kernels.
//
// Storage type S is float (the FP32 plain path) or __half (the FP16-storage
// path). All arithmetic is FP32; S only sets what the planes hold in HBM.
// Image semantics shared with the CPU oracle: reads outside the image clamp
// to the edge; bilinear sampling is exact FP32 interpolation at texel-space
// position (x, y) with texel centres on integers, clamp-to-edge (the
// reference's sampler(filter::linear) with normalised coordinates,
// demosaic.metal:146).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace gls {

template <class S>
struct is_half : std::is_same<S, __half> {};

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }

template <class S>
__device__ __forceinline__ S from_f(float v);
template <>
__device__ __forceinline__ float from_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }

// 4-channel pixel load/store (RGBA / YCbCr+w), vectorised per storage type.
struct f4 {
    float x, y, z, w;
};
struct f2 {
    float x, y;
};

template <class S>
__device__ __forceinline__ f4 ld4(const S* p);
template <>
__device__ __forceinline__ f4 ld4<float>(const float* p) {
    float4 v = *reinterpret_cast<const float4*>(p);
    return {v.x, v.y, v.z, v.w};
}
template <>
__device__ __forceinline__ f4 ld4<__half>(const __half* p) {
    uint2 u = *reinterpret_cast<const uint2*>(p);
    __half2 a = *reinterpret_cast<__half2*>(&u.x), b = *reinterpret_cast<__half2*>(&u.y);
    float2 fa = __half22float2(a), fb = __half22float2(b);
    return {fa.x, fa.y, fb.x, fb.y};
}
template <class S>
__device__ __forceinline__ void st4(S* p, f4 v);
template <>
__device__ __forceinline__ void st4<float>(float* p, f4 v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.x, v.y, v.z, v.w);
}
template <>
__device__ __forceinline__ void st4<__half>(__half* p, f4 v) {
    __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
    uint2 u;
    u.x = *reinterpret_cast<uint32_t*>(&a);
    u.y = *reinterpret_cast<uint32_t*>(&b);
    *reinterpret_cast<uint2*>(p) = u;
}
template <class S>
__device__ __forceinline__ f2 ld2(const S* p);
template <>
__device__ __forceinline__ f2 ld2<float>(const float* p) {
    float2 v = *reinterpret_cast<const float2*>(p);
    return {v.x, v.y};
}
template <>
__device__ __forceinline__ f2 ld2<__half>(const __half* p) {
    float2 v = __half22float2(*reinterpret_cast<const __half2*>(p));
    return {v.x, v.y};
}
template <class S>
__device__ __forceinline__ void st2(S* p, f2 v);
template <>
__device__ __forceinline__ void st2<float>(float* p, f2 v) {
    *reinterpret_cast<float2*>(p) = make_float2(v.x, v.y);
}
template <>
__device__ __forceinline__ void st2<__half>(__half* p, f2 v) {
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(v.x, v.y);
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.f, 1.f);
    return t * t * (3.f - 2.f * t);
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a + (b - a) * t; }

// Bayer offsets (x, y) of R, G, B, G2 per pattern, demosaic.metal:33-38.
__constant__ static const int8_t kBayer[4][4][2] = {
    {{1, 0}, {0, 0}, {0, 1}, {1, 1}},
    {{0, 1}, {0, 0}, {1, 0}, {1, 1}},
    {{0, 0}, {0, 1}, {1, 1}, {1, 0}},
    {{1, 1}, {0, 1}, {0, 0}, {1, 0}},
};

__device__ __forceinline__ int bayer_channel(int pattern, int x, int y) {
    int c = 0;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (kBayer[pattern][k][0] == (x & 1) && kBayer[pattern][k][1] == (y & 1)) c = k;
    return c;
}

// A 2-D plane in device memory: C interleaved channels of S, pitch in
// elements of S.
template <class S, int C>
struct Plane {
    S* p;
    int w, h;
    size_t pitch;  // elements per row
    __device__ __forceinline__ S* px(int x, int y) const { return p + size_t(y) * pitch + size_t(x) * C; }
    __device__ __forceinline__ S* pxc(int x, int y) const { return px(clampi(x, 0, w - 1), clampi(y, 0, h - 1)); }
};

}  // namespace gls
