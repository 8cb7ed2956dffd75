// gls_gray.cu — convertToGrayscale (demosaic.metal:1707-1723): the luma
// image PyramidFusion's main_full registers on (convertImage,
// pyramidFusion.cpp:80-98): max(t . ((rgb - 0.1) / 0.9), 0), one rounding
// per operation in the reference's order.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/glscam.h"
#include "gls_host.h"

namespace {
template <class S>
__device__ __forceinline__ float ldf(const S* p, int c);
template <>
__device__ __forceinline__ float ldf<float>(const float* p, int c) { return p[c]; }
template <>
__device__ __forceinline__ float ldf<__half>(const __half* p, int c) { return __half2float(p[c]); }

template <class S>
__global__ void k_gray(const S* __restrict__ in, size_t in_pitch, int w, int h, float t0, float t1, float t2,
                       float* __restrict__ out, size_t out_pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const S* p = in + size_t(y) * in_pitch + size_t(x) * 4;
    const float r = __fdiv_rn(__fsub_rn(ldf(p, 0), 0.1f), 0.9f);
    const float g = __fdiv_rn(__fsub_rn(ldf(p, 1), 0.1f), 0.9f);
    const float b = __fdiv_rn(__fsub_rn(ldf(p, 2), 0.1f), 0.9f);
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(t0, r), __fmul_rn(t1, g)), __fmul_rn(t2, b));
    out[size_t(y) * out_pitch + x] = fmaxf(d, 0.f);
}
}  // namespace

using namespace gls;

extern "C" gls_status gls_convert_to_grayscale(const gls_image_view* rgb, const float* transform,
                                               gls_image_view* gray, void* stream) {
    clear_error();
    if (!rgb || !gray || !transform || !rgb->data || !gray->data) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (rgb->channels != 4) return set_error(GLS_ERR_INVALID_ARG, "the RGB view must have 4 channels");
    if (gray->channels != 1 || gray->dtype != GLS_F32) return set_error(GLS_ERR_INVALID_ARG, "the output must be 1-channel F32");
    if (gray->width != rgb->width || gray->height != rgb->height) return set_error(GLS_ERR_INVALID_ARG, "size mismatch");
    const size_t es = rgb->dtype == GLS_F32 ? 4 : rgb->dtype == GLS_F16 ? 2 : 0;
    if (!es) return set_error(GLS_ERR_INVALID_ARG, "RGB dtype must be F32 or F16");
    if (rgb->stride_bytes % (4 * es) || gray->stride_bytes % 4)
        return set_error(GLS_ERR_INVALID_ARG, "strides must be whole pixels");
    const int w = rgb->width, h = rgb->height;
    if (w <= 0 || h <= 0) return set_error(GLS_ERR_INVALID_ARG, "empty image");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
    if (es == 4)
        k_gray<float><<<g, b, 0, s>>>(static_cast<const float*>(rgb->data), rgb->stride_bytes / 4, w, h, transform[0],
                                     transform[1], transform[2], static_cast<float*>(gray->data), gray->stride_bytes / 4);
    else
        k_gray<__half><<<g, b, 0, s>>>(static_cast<const __half*>(rgb->data), rgb->stride_bytes / 2, w, h, transform[0],
                                      transform[1], transform[2], static_cast<float*>(gray->data), gray->stride_bytes / 4);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "convertToGrayscale launch: %s", cudaGetErrorString(e));
    return GLS_OK;
}
