// gls_host.h — host-side helpers shared by the C-ABI translation units.
#pragma once

#include "../../include/glscam.h"

namespace gls {

// Record an error message for gls_last_error_message() and return code.
gls_status set_error(gls_status code, const char* fmt, ...);
void clear_error();

gls_status calibration_fill(int camera, int iso, gls_demosaic_params* p);
// Fills (weight, dx, dy) taps; returns the tap count, or -count if max_taps
// is too small.
int gaussian_taps(float radius, float* out, int max_taps);
void cam_ycbcr(const float rgb_cam[9], const float xyz_rgb[9], float fwd[9], float inv[9]);

}  // namespace gls
