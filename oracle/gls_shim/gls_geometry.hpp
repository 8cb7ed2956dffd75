// gls_geometry.hpp — TEST INFRASTRUCTURE ONLY. Stand-in for the GlassImage
// geometry helper the reference's Homography.cpp calls (applyHomography).
// The projected point is ((h00 x + h01 y) + h02, (h10 x + h11 y) + h12)
// divided by (h20 x + h21 y) + h22, one rounding per operation, as the
// registration oracle reads it.
#pragma once

#include "gls_image.hpp"
#include "gls_linalg.hpp"

namespace gls {

inline basic_point<float> applyHomography(const basic_point<float>& p, const Matrix<3, 3>& H) {
    const float w = H[2][0] * p.x + H[2][1] * p.y + H[2][2];
    return {(H[0][0] * p.x + H[0][1] * p.y + H[0][2]) / w, (H[1][0] * p.x + H[1][1] * p.y + H[1][2]) / w};
}

}  // namespace gls
