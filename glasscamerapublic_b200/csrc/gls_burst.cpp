// gls_burst.cpp — the host side of the burst driver around the GPU path
// (PyramidFusion/pyramidFusion.cpp): grouping a directory's frames into
// bursts (findBursts, :166-195) and writing the fused image as an 8-bit RGB
// TIFF (saveFusedImage, :152-164).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/glscam.h"
#include "gls_host.h"

using namespace gls;

namespace {
// the file name without directory and extension (std::filesystem::path::stem)
std::string stem_of(const char* path) {
    std::string s(path);
    const size_t slash = s.find_last_of('/');
    if (slash != std::string::npos) s = s.substr(slash + 1);
    if (s == "." || s == "..") return s;
    const size_t dot = s.find_last_of('.');
    if (dot != std::string::npos && dot > 0) s = s.substr(0, dot);
    return s;
}
}  // namespace

extern "C" gls_status gls_find_bursts(const char* const* paths, int32_t n, int32_t* burst_of, int32_t* n_bursts) {
    clear_error();
    if ((!paths || !burst_of) && n > 0) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (n < 0) return set_error(GLS_ERR_INVALID_ARG, "negative count");
    // a stem containing "_1_" starts a burst; later files join it when their
    // stem has the same prefix up to that position; files before any start,
    // or with another prefix, belong to none
    int current = -1;
    std::string prefix;
    size_t found = std::string::npos;
    for (int i = 0; i < n; i++) {
        burst_of[i] = -1;
        if (!paths[i]) continue;
        const std::string st = stem_of(paths[i]);
        const size_t f = st.find("_1_");
        if (f != std::string::npos) {
            current++;
            found = f;
            prefix = st.substr(0, f);
            burst_of[i] = current;
        } else if (found != std::string::npos && st.substr(0, found) == prefix) {
            burst_of[i] = current;
        }
    }
    if (n_bursts) *n_bursts = current + 1;
    return GLS_OK;
}

extern "C" gls_status gls_write_tiff_rgb8(const char* path, const gls_image_view* rgba, void* stream) {
    clear_error();
    if (!path || !rgba || !rgba->data) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (rgba->channels < 3) return set_error(GLS_ERR_INVALID_ARG, "the image needs 3 or 4 channels");
    const size_t es = rgba->dtype == GLS_F32 ? 4 : rgba->dtype == GLS_F16 ? 2 : 0;
    if (!es) return set_error(GLS_ERR_INVALID_ARG, "image dtype must be F32 or F16");
    const int W = rgba->width, H = rgba->height, C = rgba->channels;
    if (W <= 0 || H <= 0) return set_error(GLS_ERR_INVALID_ARG, "empty image");
    const size_t row = size_t(W) * C * es;
    if (rgba->stride_bytes < row) return set_error(GLS_ERR_INVALID_ARG, "stride too small");
    // the pixels in host memory (a device view is copied back first)
    std::vector<uint8_t> host(row * H);
    cudaPointerAttributes at{};
    const bool dev = cudaPointerGetAttributes(&at, rgba->data) == cudaSuccess &&
                     (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    if (dev) {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (cudaMemcpy2DAsync(host.data(), row, rgba->data, rgba->stride_bytes, row, H, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return set_error(GLS_ERR_CUDA, "copying the image to the host failed");
    } else {
        for (int y = 0; y < H; y++)
            std::memcpy(&host[row * y], static_cast<const uint8_t*>(rgba->data) + rgba->stride_bytes * y, row);
    }
    // (uint8_t) (255 * clamp(v, 0, 1)) per channel (pyramidFusion.cpp:155-160)
    std::vector<uint8_t> rgb(size_t(W) * H * 3);
    for (size_t i = 0; i < size_t(W) * H; i++)
        for (int c = 0; c < 3; c++) {
            float v;
            if (es == 4) {
                std::memcpy(&v, &host[(i * C + c) * 4], 4);
            } else {
                __half h;
                std::memcpy(&h, &host[(i * C + c) * 2], 2);
                v = __half2float(h);
            }
            rgb[i * 3 + c] = uint8_t(255 * std::clamp(v, 0.0f, 1.0f));
        }
    // an uncompressed little-endian RGB TIFF, one strip
    std::vector<uint8_t> t = {'I', 'I', 42, 0, 8, 0, 0, 0};
    auto u16 = [&](uint16_t v) { t.push_back(uint8_t(v)), t.push_back(uint8_t(v >> 8)); };
    auto u32 = [&](uint32_t v) { for (int k = 0; k < 4; k++) t.push_back(uint8_t(v >> (8 * k))); };
    const uint16_t n_entries = 10;
    const uint32_t bps_at = 8 + 2 + 12 * n_entries + 4, data_at = bps_at + 8;
    u16(n_entries);
    auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
        u16(tag), u16(type), u32(count);
        if (type == 3 && count == 1) u16(uint16_t(value)), u16(0);
        else u32(value);
    };
    entry(256, 4, 1, uint32_t(W));           // ImageWidth
    entry(257, 4, 1, uint32_t(H));           // ImageLength
    entry(258, 3, 3, bps_at);                // BitsPerSample 8, 8, 8
    entry(259, 3, 1, 1);                     // no compression
    entry(262, 3, 1, 2);                     // RGB
    entry(273, 4, 1, data_at);               // StripOffsets
    entry(277, 3, 1, 3);                     // SamplesPerPixel
    entry(278, 4, 1, uint32_t(H));           // RowsPerStrip
    entry(279, 4, 1, uint32_t(rgb.size()));  // StripByteCounts
    entry(284, 3, 1, 1);                     // PlanarConfiguration: contiguous
    u32(0);
    u16(8), u16(8), u16(8), u16(0);
    t.insert(t.end(), rgb.begin(), rgb.end());
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_error(GLS_ERR_INVALID_ARG, "cannot write %s", path);
    const size_t put = std::fwrite(t.data(), 1, t.size(), f);
    std::fclose(f);
    if (put != t.size()) return set_error(GLS_ERR_INVALID_ARG, "short write to %s", path);
    return GLS_OK;
}
