// Small fixed-size dense linear algebra used by the host-side mesh setup and
// by the output diagnostics: the operations the reference takes from Eigen 3
// (not available here), restated from their textbook definitions.
//
//   * full-pivoting LU rank test      (Eigen::FullPivLU::isInvertible,
//                                       used at set_up_patch_fitting.cpp:227)
//   * inverse via LU with partial pivoting (Matrix<6,6>::inverse(),
//                                       set_up_patch_fitting.cpp:232)
//   * 3x3 inverse via cofactors        (Matrix3d::inverse(), calc_deriv_mats.cpp:78-90)
//   * largest singular value of a 6x3 (JacobiSVD::singularValues()(0),
//                                       set_up_patch_fitting.cpp:243)
//   * symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations
//                                      (SelfAdjointEigenSolver, calc_stresses.cpp:162)
//
// The routines compile for the host and, under nvcc, for the device as well
// (the device set-up in setup.cu): the same operations in the same order,
// so with contraction into fused multiply-adds off on the device both give
// the same bits.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define MSB_HD __host__ __device__
#else
#define MSB_HD
#endif

namespace msb {
namespace la {

template <typename T>
MSB_HD inline void swap_values(T& a, T& b) {
    T t = a;
    a = b;
    b = t;
}

// The machine epsilon of double (std::numeric_limits<double>::epsilon()).
constexpr double kEpsilon = 2.220446049250313080847e-16;

// Rank of an n x n matrix (row-major, copied) by Gaussian elimination with
// complete pivoting.  A pivot counts as non-zero when its magnitude exceeds
// n * eps * (largest pivot met), the default threshold of a full-pivoting LU.
template <int N>
MSB_HD inline int full_piv_rank(const double (&a_in)[N][N]) {
    double a[N][N];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) a[i][j] = a_in[i][j];
    double pivots[N];
    int npiv = N;
    double maxpivot = 0.0;
    for (int k = 0; k < N; ++k) {
        int bi = k, bj = k;
        double best = -1.0;
        for (int i = k; i < N; ++i)
            for (int j = k; j < N; ++j)
                if (fabs(a[i][j]) > best) { best = fabs(a[i][j]); bi = i; bj = j; }
        if (best == 0.0) {
            npiv = k;
            break;
        }
        if (best > maxpivot) maxpivot = best;
        if (bi != k) for (int j = 0; j < N; ++j) swap_values(a[k][j], a[bi][j]);
        if (bj != k) for (int i = 0; i < N; ++i) swap_values(a[i][k], a[i][bj]);
        pivots[k] = a[k][k];
        for (int i = k + 1; i < N; ++i) {
            double f = a[i][k] / a[k][k];
            for (int j = k + 1; j < N; ++j) a[i][j] -= f * a[k][j];
            a[i][k] = 0.0;
        }
    }
    const double thresh = maxpivot * kEpsilon * N;
    int rank = 0;
    for (int k = 0; k < npiv; ++k)
        if (fabs(pivots[k]) > thresh) ++rank;
    return rank;
}

// Inverse of an n x n matrix by LU with partial (row) pivoting; returns false
// when a pivot is exactly zero.
template <int N>
MSB_HD inline bool inverse_partial_piv(const double (&a_in)[N][N], double (&inv)[N][N]) {
    double lu[N][N];
    int perm[N];
    for (int i = 0; i < N; ++i) {
        perm[i] = i;
        for (int j = 0; j < N; ++j) lu[i][j] = a_in[i][j];
    }
    for (int k = 0; k < N; ++k) {
        int p = k;
        double best = fabs(lu[k][k]);
        for (int i = k + 1; i < N; ++i)
            if (fabs(lu[i][k]) > best) { best = fabs(lu[i][k]); p = i; }
        if (best == 0.0) return false;
        if (p != k) {
            for (int j = 0; j < N; ++j) swap_values(lu[k][j], lu[p][j]);
            swap_values(perm[k], perm[p]);
        }
        for (int i = k + 1; i < N; ++i) {
            lu[i][k] /= lu[k][k];
            for (int j = k + 1; j < N; ++j) lu[i][j] -= lu[i][k] * lu[k][j];
        }
    }
    // Solve L U x = P e_c for each column c of the identity.
    for (int c = 0; c < N; ++c) {
        double x[N];
        for (int i = 0; i < N; ++i) x[i] = (perm[i] == c) ? 1.0 : 0.0;
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < i; ++j) x[i] -= lu[i][j] * x[j];
        for (int i = N - 1; i >= 0; --i) {
            for (int j = i + 1; j < N; ++j) x[i] -= lu[i][j] * x[j];
            x[i] /= lu[i][i];
        }
        for (int i = 0; i < N; ++i) inv[i][c] = x[i];
    }
    return true;
}

// 3x3 inverse by the adjugate: inv = adj(a) / det(a).
MSB_HD inline void inverse3(const double (&a)[3][3], double (&inv)[3][3]) {
    double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    double id = 1.0 / det;
    inv[0][0] = c00 * id;
    inv[1][0] = c01 * id;
    inv[2][0] = c02 * id;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) * id;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) * id;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) * id;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) * id;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) * id;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) * id;
}

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations.
// Eigenvalues come out in ascending order; column k of vecs is the unit
// eigenvector of vals[k].
MSB_HD inline void sym_eig3(const double (&a_in)[3][3], double (&vals)[3], double (&vecs)[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            a[i][j] = 0.5 * (a_in[i][j] + a_in[j][i]);
            vecs[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 64; ++sweep) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        double diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off <= 1e-36 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    double vkp = vecs[k][p], vkq = vecs[k][q];
                    vecs[k][p] = c * vkp - s * vkq;
                    vecs[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) vals[i] = a[i][i];
    // Sort ascending, permuting eigenvector columns alongside.
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2 - i; ++j)
            if (vals[j] > vals[j + 1]) {
                swap_values(vals[j], vals[j + 1]);
                for (int k = 0; k < 3; ++k) swap_values(vecs[k][j], vecs[k][j + 1]);
            }
}

// Largest singular value of a 6x3 matrix: sqrt of the largest eigenvalue of
// its 3x3 Gram matrix.
MSB_HD inline double max_singular_value_6x3(const double (&m)[6][3]) {
    double g[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 6; ++k) s += m[k][i] * m[k][j];
            g[i][j] = s;
        }
    double vals[3], vecs[3][3];
    sym_eig3(g, vals, vecs);
    return sqrt(vals[2] < 0.0 ? 0.0 : vals[2]);  // std::max(vals[2], 0.0), NaN kept
}

}  // namespace la
}  // namespace msb
