// ref_reg_metal.h — TEST INFRASTRUCTURE ONLY. Plain-typed entry points into
// the reference's SURF.metal kernels compiled for the CPU
// (ref_reg_metal.cpp), called per thread by ref_reg_harness.cpp. The Metal
// source is compiled in a translation unit of its own because Metal has no
// double: its unsuffixed floating literals are float
// (-fsingle-precision-constant), while the host C++ of SURF.cpp keeps
// double literals.
#pragma once

#include <metal_stdlib>

// the shim's address-space keywords are for Metal source only
#undef kernel
#undef device
#undef thread
#undef threadgroup
#undef constant

namespace refwrap {

struct KeyPoint {  // SURF.metal:179-187
    float x, y, size, angle, response;
    int octave, class_id;
};
constexpr int kMaximaCapacity = 64000;  // KeyPointMaxima_MaxCount, SURF.metal:249
struct Maxima {                         // KeyPointMaxima, SURF.metal:250-253
    int count;
    KeyPoint kp[kMaximaCapacity];
};
struct Match {  // DMatch, SURF.metal:430-434
    unsigned query_idx, train_idx;
    float distance;
};

void integral_sum_cols(metal::tex_store* src, float* buf, int buf_width, unsigned lid, unsigned gid, unsigned x);
void integral_sum_rows(float* buf, int buf_width, metal::tex_store* s0, metal::tex_store* s1, metal::tex_store* s2,
                       metal::tex_store* s3, unsigned lid, unsigned gid, unsigned gs, unsigned x);
// surf_hf: the 256-byte SurfHF block (SURF.cpp gpuSurfHF)
void calc_det_and_trace(metal::tex_store* sum, metal::tex_store* det, metal::tex_store* trace, int step, float wx,
                        float wy, int mx, int my, const void* surf_hf, unsigned x, unsigned y);
void find_maxima_in_layer(metal::tex_store* d0, metal::tex_store* d1, metal::tex_store* d2, metal::tex_store* trace,
                          int s0, int s1, int s2, Maxima* out, int margin, int octave, float threshold, int step,
                          unsigned x, unsigned y);
// descriptors: rows of 64 floats
void match_key_points(const float* d1, const float* d2, unsigned n2, Match* out, unsigned lid, unsigned i);
void register_and_fuse(metal::tex_store* fused, metal::tex_store* input, metal::tex_store* out, const float* h9,
                       int count, unsigned x, unsigned y);

}  // namespace refwrap
