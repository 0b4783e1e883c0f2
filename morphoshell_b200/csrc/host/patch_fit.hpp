// The arithmetic of one triangle's patch fit and derivative weights, shared
// by the host set-up (mesh_setup.cpp) and the device set-up (setup.cu): the
// same operations in the same order on both sides (the device compiles them
// without fused multiply-adds), so both give the same bits.
#pragma once

#include <cmath>

#include "small_linalg.hpp"

namespace msb {
namespace patch {

// Distance of a candidate patch node from the triangle's centroid
// (set_up_patch_fitting.cpp:100-160).
MSB_HD inline double centroid_distance(const double* p, const double* centroid) {
    const double x = p[0] - centroid[0], y = p[1] - centroid[1], z = p[2] - centroid[2];
    return sqrt(x * x + y * y + z * z);
}

// One candidate patch (set_up_patch_fitting.cpp:196-262): the six nodes'
// reference positions pos[n][3] (vertices first), the triangle's centroid.
// Builds the 6x6 quadratic-fit matrix, and when it is invertible and its
// second-derivative block (the last three columns of the inverse) scaled by
// the patch size squared is better conditioned than thresh, writes the block
// and returns true.
MSB_HD inline bool try_patch(const double (&pos)[6][3], const double* centroid, double thresh,
                             double (&block)[6][3]) {
    double sq = 0.0;
    for (int n = 0; n < 6; ++n) {
        const double dx = pos[n][0] - centroid[0], dy = pos[n][1] - centroid[1], dz = pos[n][2] - centroid[2];
        sq += dx * dx + dy * dy + dz * dz;
    }
    const double patch_size = sqrt(sq / 6.0);
    double m[6][6];
    for (int n = 0; n < 6; ++n) {
        const double dx = pos[n][0] - centroid[0];
        const double dy = pos[n][1] - centroid[1];
        m[0][n] = 1.0;
        m[1][n] = dx;
        m[2][n] = dy;
        m[3][n] = 0.5 * dx * dx;
        m[4][n] = dx * dy;
        m[5][n] = 0.5 * dy * dy;
    }
    if (la::full_piv_rank<6>(m) != 6) return false;
    double inv[6][6];
    if (!la::inverse_partial_piv<6>(m, inv)) return false;
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 3; ++c) block[r][c] = inv[r][3 + c];
    const double sigma = la::max_singular_value_6x3(block);
    const double ratio = sigma * patch_size * patch_size / thresh;
    return ratio < 1.0;
}

// First-derivative weights of the three vertices (calc_deriv_mats.cpp:70-96):
// rows 1 and 2 of the inverse of the linear-interpolation matrix at the
// centroid; c[0..2] d/dx, c[3..5] d/dy.
MSB_HD inline void first_derivative_weights(const double (&vpos)[3][3], const double* centroid, double* c) {
    double a[3][3], inv[3][3];
    for (int v = 0; v < 3; ++v) {
        a[v][0] = 1.0;
        a[v][1] = vpos[v][0] - centroid[0];
        a[v][2] = vpos[v][1] - centroid[1];
    }
    la::inverse3(a, inv);
    for (int v = 0; v < 3; ++v) {
        c[v] = inv[1][v];
        c[3 + v] = inv[2][v];
    }
}

}  // namespace patch
}  // namespace msb
