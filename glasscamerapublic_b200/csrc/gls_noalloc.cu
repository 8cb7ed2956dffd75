// gls_noalloc.cu — gls_pca_basis_noalloc: the PCA patch basis of one image
// (the per-level collectPatches + covariance + eigen-solve of the pyramid
// denoise) computed without allocating any device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they
// need the basis. A camera pipeline's real-time capture thread must not
// block in the allocator (cudaMalloc can synchronise the device and take
// milliseconds), and an application whose device memory is entirely handed
// out by another framework's caching allocator has no room for a second
// allocator. Such a caller passes its own input image and output basis; the
// only other memory the computation needs (the per-chunk covariance
// partials) lives in the fixed array below, which every GPU that loads this
// library holds until the process exits.
#include <mutex>

#include "gls_common.cuh"
#include "gls_host.h"
#include "gls_kernels.h"

namespace gls {

// Covariance partial sums: one row of kPcaAcc FP64 sums per 64-patch chunk.
// 4096 rows = 11.5 MB, so at most 4096 x 64 = 262,144 patches per image
// (an image of at most ~16.7 megapixels, e.g. 4096 x 4096 or 4032 x 3024).
constexpr int kNoAllocRows = 4096;
constexpr long kNoAllocMaxPatches = long(kNoAllocRows) * kPcaChunk;

static __device__ __align__(256) double g_pca_partials[kNoAllocRows * kPcaAcc];

// Device address of g_pca_partials, looked up once per device (host code
// cannot use the symbol itself: on the host it names a stand-in, not device
// memory).
static std::mutex g_setup_mutex;
static void* g_partials_ptr[64] = {};

static gls_status partials_address(int device, double** out) {
    if (device < 0 || device >= 64) return set_error(GLS_ERR_INVALID_ARG, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_pca_partials);
        if (e != cudaSuccess || !p)
            return set_error(GLS_ERR_CUDA, "cudaGetSymbolAddress(g_pca_partials) failed on device %d: %s", device,
                             cudaGetErrorString(e));
        g_partials_ptr[device] = p;
    }
    *out = static_cast<double*>(g_partials_ptr[device]);
    return GLS_OK;
}

}  // namespace gls

using namespace gls;

extern "C" gls_status gls_pca_basis_noalloc(const gls_image_view* image, float* basis25x8, void* stream) {
    clear_error();
    if (!image || !image->data || !basis25x8) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (image->channels != 4) return set_error(GLS_ERR_INVALID_ARG, "image must have 4 channels (luma first)");
    if (image->dtype != GLS_F32 && image->dtype != GLS_F16)
        return set_error(GLS_ERR_INVALID_ARG, "image dtype must be GLS_F32 or GLS_F16");
    if (image->width < 1 || image->height < 1) return set_error(GLS_ERR_INVALID_ARG, "empty image");
    const size_t es = image->dtype == GLS_F32 ? 4 : 2;
    if (image->stride_bytes < size_t(image->width) * 4 * es || image->stride_bytes % (4 * es) ||
        uintptr_t(image->data) % (4 * es))
        return set_error(GLS_ERR_INVALID_ARG, "image rows must be %zu-byte aligned with a matching stride", 4 * es);
    const long patches = long(image->width / 8) * long(image->height / 8);
    if (patches > kNoAllocMaxPatches)
        return set_error(GLS_ERR_INVALID_ARG,
                         "image %dx%d has %ld PCA patches; gls_pca_basis_noalloc holds at most %ld "
                         "(its fixed scratch has %d rows of 64 patches)",
                         image->width, image->height, patches, kNoAllocMaxPatches, kNoAllocRows);
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    double* part = nullptr;
    gls_status st = partials_address(device, &part);
    if (st != GLS_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // every row the eigen kernel reads is rewritten by the covariance kernel
    // of this call, so nothing has to be cleared first
    const int rows = int((patches + kPcaChunk - 1) / kPcaChunk);
    if (image->dtype == GLS_F32) {
        Plane<float, 4> img{static_cast<float*>(image->data), image->width, image->height, image->stride_bytes / 4};
        launch_pca_cov_rows<float>(img, part, rows, s);
    } else {
        Plane<__half, 4> img{static_cast<__half*>(image->data), image->width, image->height, image->stride_bytes / 2};
        launch_pca_cov_rows<__half>(img, part, rows, s);
    }
    launch_pca_eigen(part, rows, int(patches), basis25x8, nullptr, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GLS_ERR_CUDA, "launch failed: %s", cudaGetErrorString(e));
    return GLS_OK;
}
