// gls_noise.h — the grain tables of convertTosRGB (Noise2D::randomSeed +
// initGradients, SimplexNoise.hpp:109-143, B = 256), host and device.
//
// The reference draws them from the C library: srandom(seed), then
// random(). Both the GNU and the BSD C libraries implement random() as the
// same additive-feedback generator of degree 31 (r[i] = r[i-31] + r[i-3]
// mod 2^32, output r[i] >> 1) seeded by the Park-Miller recurrence
// r[i] = 16807 r[i-1] mod (2^31 - 1), with the first 310 outputs
// discarded. They differ only for seed 0 (the GNU library uses 1, the BSD
// library 123459876); this restatement follows the GNU library, which the
// tests pin it against.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define GLS_NOISE_HD __host__ __device__
#else
#define GLS_NOISE_HD
#endif

namespace gls {

constexpr int kNoiseSize = 514;  // 2 * 256 + 2 entries

struct RandomR {
    uint32_t r[34];
    int i = 0;  // ring position of r[n]
    GLS_NOISE_HD explicit RandomR(uint32_t seed) {
        int32_t word = seed == 0 ? 1 : int32_t(seed);
        r[0] = uint32_t(word);
        for (int k = 1; k < 31; k++) {
            const int32_t hi = word / 127773, lo = word % 127773;
            word = 16807 * lo - 2836 * hi;
            if (word < 0) word += 2147483647;
            r[k] = uint32_t(word);
        }
        for (int k = 31; k < 34; k++) r[k] = r[k - 31];
        i = 0;
        for (int k = 0; k < 310; k++) next();
    }
    // the generator step: r[n] = r[n-31] + r[n-3], returned >> 1
    GLS_NOISE_HD int32_t next() {
        // ring of 34 entries: r[n-34] sits at slot i; r[n-31] at i + 3; r[n-3] at i + 31
        const uint32_t v = r[(i + 3) % 34] + r[(i + 31) % 34];
        r[i] = v;
        i = (i + 1) % 34;
        return int32_t(v >> 1);
    }
};

// perm[514], grad[514][2]
GLS_NOISE_HD inline void noise_tables(uint32_t seed, int* perm, float* grad) {
    RandomR rnd(seed);
    for (int i = 0; i < 256; i++) {
        perm[i] = i;
        for (int j = 0; j < 2; j++) grad[2 * i + j] = float((rnd.next() % 512) - 256) / 256;
        const float s = sqrtf(grad[2 * i] * grad[2 * i] + grad[2 * i + 1] * grad[2 * i + 1]);
        grad[2 * i] = grad[2 * i] / s;
        grad[2 * i + 1] = grad[2 * i + 1] / s;
    }
    for (int i = 255; i > 0; i--) {
        const int k = perm[i];
        const int j = rnd.next() % 256;
        perm[i] = perm[j];
        perm[j] = k;
    }
    for (int i = 0; i < 258; i++) {
        perm[256 + i] = perm[i];
        grad[2 * (256 + i)] = grad[2 * i];
        grad[2 * (256 + i) + 1] = grad[2 * i + 1];
    }
}

}  // namespace gls
