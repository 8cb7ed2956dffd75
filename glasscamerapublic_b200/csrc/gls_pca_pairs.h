// gls_pca_pairs.h — index map of the PCA covariance accumulators.
//
// The 25x25 patch covariance is symmetric, so the accumulators hold its
// upper triangle: entry (r, c), r <= c, at index r*25 - r*(r-1)/2 + (c - r)
// (row-major over the triangle, 325 entries), followed by the 25 component
// sums. pca_pair() is the inverse, used by the covariance kernel to find
// the entry a thread owns. It is computed from the thread index, so no
// per-device table has to be loaded before the kernel runs. Plain C++ with
// host/device qualifiers only under nvcc, so the same code is compiled by
// the host compiler in the CPU tests.
#pragma once

#if defined(__CUDACC__)
#define GLS_HD __host__ __device__
#else
#define GLS_HD
#endif

namespace gls {

constexpr int kPcaTri = 325;  // upper-triangle entries of a 25x25 matrix

GLS_HD constexpr int pca_tri_index(int r, int c) { return r * 25 - r * (r - 1) / 2 + (c - r); }

// (r, c) of upper-triangle index t in [0, 325): rows hold 25, 24, ..., 1
// entries, so subtract row lengths until t falls inside one.
GLS_HD constexpr void pca_pair(int t, int& r, int& c) {
    int row = 0, rem = t;
    while (row < 24 && rem >= 25 - row) {
        rem -= 25 - row;
        row++;
    }
    r = row;
    c = row + rem;
}

GLS_HD constexpr bool pca_pairs_consistent() {
    int k = 0;
    for (int i = 0; i < 25; i++)
        for (int j = i; j < 25; j++, k++) {
            int r = -1, c = -1;
            pca_pair(k, r, c);
            if (r != i || c != j || pca_tri_index(i, j) != k) return false;
        }
    return k == kPcaTri;
}
static_assert(pca_pairs_consistent(), "pca_pair must invert pca_tri_index on all 325 entries");

}  // namespace gls
