// ref_noise.cpp — TEST INFRASTRUCTURE ONLY. The grain tables of
// convertTosRGB drawn by the reference's own Noise2D
// (MetalPipeline/SimplexNoise.hpp, included where it lies in the reference
// tree): srandom(seed), then initGradients. A translation unit of its own,
// because the header's global mix() and s_curve() would collide with the
// Metal helpers of ref_harness.cpp. Part of _ref/libglsref.so.
#include <array>
#include <cmath>
#include <cstdlib>

#include "SimplexNoise.hpp"

extern "C" int ref_noise_tables(unsigned seed, int* perm, float* grad) {
    std::array<int, Noise2D::arraySize> p;
    std::array<std::array<float, 2>, Noise2D::arraySize> g;
    Noise2D::randomSeed(seed);
    Noise2D::initGradients(&p, &g);
    for (int i = 0; i < Noise2D::arraySize; i++) {
        perm[i] = p[i];
        grad[2 * i] = g[i][0];
        grad[2 * i + 1] = g[i][1];
    }
    return 0;
}
