// ref_reg_metal.cpp — TEST INFRASTRUCTURE ONLY. The reference's SURF.metal,
// compiled as C++ against metal_shim/, behind the plain-typed entry points
// of ref_reg_metal.h. Unmodified line ranges SURF.metal:17-40 and 64-559 are
// extracted into oracle/_ref/ by `make -C oracle ref` (not committed).
// SURF.metal:41-63 (_int8, _float8) is restated: GCC rejects class-type
// members in an anonymous struct; the restatement keeps the members and the
// layout. `threadgroup` arrays become function statics, shared by the host
// threads that run one threadgroup at a time (ref_reg_harness.cpp).
//
// SURF.metal:200 `(float3)(a, b, c)` compiles as C++ reads it, and as Metal
// (a C++14 dialect) does: a cast of the comma expression, float3(c).
#include "ref_reg_metal.h"

#include <cstring>

// MSL address-space and function qualifiers (threadgroup: see above)
#define kernel
#define device
#define thread
#define constant
#define threadgroup static

namespace refmtl {
#include "surf_metal_a.inc"

struct _int8 {  // SURF.metal:41-51
    int4 lo;
    int4 hi;
    _int8() = default;
    _int8(int val) : lo(val), hi(val) {}
};
struct _float8 {  // SURF.metal:53-63
    float4 lo;
    float4 hi;
    _float8() = default;
    _float8(float val) : lo(val), hi(val) {}
};

#include "surf_metal_b.inc"
}  // namespace refmtl

#undef kernel
#undef device
#undef thread
#undef constant
#undef threadgroup

namespace refwrap {

using metal::access;
using metal::texture2d;

static_assert(sizeof(refmtl::KeyPoint) == sizeof(KeyPoint), "KeyPoint layout");
static_assert(sizeof(refmtl::KeyPointMaxima) == sizeof(Maxima), "KeyPointMaxima layout");
static_assert(sizeof(refmtl::DMatch) == sizeof(Match), "DMatch layout");
static_assert(sizeof(refmtl::SurfHF) == 256, "SurfHF layout");
static_assert(sizeof(refmtl::array<refmtl::float4, 16>) == 64 * sizeof(float), "descriptor layout");

void integral_sum_cols(metal::tex_store* src, float* buf, int buf_width, unsigned lid, unsigned gid, unsigned x) {
    refmtl::integral_sum_cols_image(texture2d<float>(src), buf, buf_width, lid, gid, x);
}

void integral_sum_rows(float* buf, int buf_width, metal::tex_store* s0, metal::tex_store* s1, metal::tex_store* s2,
                       metal::tex_store* s3, unsigned lid, unsigned gid, unsigned gs, unsigned x) {
    refmtl::integral_sum_rows_image(buf, buf_width, texture2d<float, access::write>(s0),
                                    texture2d<float, access::write>(s1), texture2d<float, access::write>(s2),
                                    texture2d<float, access::write>(s3), lid, gid, gs, x);
}

void calc_det_and_trace(metal::tex_store* sum, metal::tex_store* det, metal::tex_store* trace, int step, float wx,
                        float wy, int mx, int my, const void* surf_hf, unsigned x, unsigned y) {
    refmtl::SurfHF hf;
    std::memcpy(&hf, surf_hf, sizeof(hf));
    refmtl::float2 w(wx, wy);
    refmtl::int2 margin(mx, my);
    refmtl::calcDetAndTrace(texture2d<float>(sum), texture2d<float, access::write>(det),
                            texture2d<float, access::write>(trace), step, w, margin, &hf, refmtl::uint2(x, y));
}

void find_maxima_in_layer(metal::tex_store* d0, metal::tex_store* d1, metal::tex_store* d2, metal::tex_store* trace,
                          int s0, int s1, int s2, Maxima* out, int margin, int octave, float threshold, int step,
                          unsigned x, unsigned y) {
    refmtl::int3 sizes(s0, s1, s2);
    refmtl::findMaximaInLayer(texture2d<float>(d0), texture2d<float>(d1), texture2d<float>(d2),
                              texture2d<float>(trace), sizes, reinterpret_cast<refmtl::KeyPointMaxima*>(out),
                              margin, octave, threshold, step, refmtl::uint2(x, y));
}

void match_key_points(const float* d1, const float* d2, unsigned n2, Match* out, unsigned lid, unsigned i) {
    using Row = refmtl::array<refmtl::float4, 16>;
    refmtl::matchKeyPoints(reinterpret_cast<Row*>(const_cast<float*>(d1)),
                           reinterpret_cast<Row*>(const_cast<float*>(d2)), n2,
                           reinterpret_cast<refmtl::DMatch*>(out), refmtl::uint2(0, lid), refmtl::uint2(i, lid));
}

void register_and_fuse(metal::tex_store* fused, metal::tex_store* input, metal::tex_store* out, const float* h9,
                       int count, unsigned x, unsigned y) {
    refmtl::Matrix3x3 m;
    for (int i = 0; i < 3; i++) m.m[i] = refmtl::float3(h9[3 * i], h9[3 * i + 1], h9[3 * i + 2]);
    refmtl::registerAndFuse(texture2d<float>(fused), texture2d<float>(input), texture2d<float, access::write>(out),
                            m, count, refmtl::uint2(x, y));
}

}  // namespace refwrap
