// Per-triangle force contributions over the per-triangle (AoS) tables,
// shared by the two-kernel, cluster-tiled and batched steps.
#pragma once

#include "internal.cuh"
#include "tri_physics.cuh"

namespace msb {
namespace tridev {

using dev::Cq;
using dev::CqGrad;
using dev::TriMat;

template <bool MIXED>
struct Real {
    using T = double;
};
template <>
struct Real<true> {
    using T = float;
};

// Contributions of triangle t to its six patch nodes, in the precision of
// the path (double, or float for the mixed path).
template <int DIAL, bool MIXED>
__device__ __forceinline__ void tri_contrib(const DevMesh& m, const ClusterPlan& p, const double* __restrict__ pos,
                                            int t, const int (&ids)[6], double dial, double lam, double pw,
                                            typename Real<MIXED>::T (&f)[18], double nu, double gamma) {
    using R = typename Real<MIXED>::T;
    const int N = m.N;
    TriMat<double> mt;
    if (m.uniform_hmu) {
        mt.h = m.h_uniform;
        mt.mu = m.mu_uniform;
    } else {
        mt.h = __ldg(m.thick + t);
        mt.mu = __ldg(m.shear + t);
    }
    if (DIAL == DIAL_LCE) {
        const double2* ap = reinterpret_cast<const double2*>(p.tri_aux + t);
        const double2 a01 = __ldg(ap), a23 = __ldg(ap + 1);
        const double4 aux = {a01.x, a01.y, a23.x, a23.y};
        mt.area = aux.x;
        double l2 = lam * lam, pp = pw;
        if (!p.lce_uniform) {
            const double2 ln = __ldg(p.lce_ln + t);
            const double lt = (1.0 - dial) * 1.0 + dial * ln.x;
            l2 = lt * lt;
            pp = pow(lt, -2.0 * ln.y);
        }
        mt.abar0 = l2 * aux.y + pp * aux.z;
        mt.abar1 = (l2 - pp) * aux.w;
        mt.abar2 = pp * aux.y + l2 * aux.z;
        mt.bbar0 = mt.bbar1 = mt.bbar2 = 0.0;
    } else {
        mt.area = __ldg(m.area + t);
        mt.abar0 = __ldg(m.abar + t);
        mt.abar1 = __ldg(m.abar + (size_t)m.T + t);
        mt.abar2 = __ldg(m.abar + 2 * (size_t)m.T + t);
        mt.bbar0 = __ldg(m.bbar + t);
        mt.bbar1 = __ldg(m.bbar + (size_t)m.T + t);
        mt.bbar2 = __ldg(m.bbar + 2 * (size_t)m.T + t);
    }
    R c[24];
    if constexpr (!MIXED) {
        const double2* cp = reinterpret_cast<const double2*>(p.coef_aos + 24 * (size_t)t);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            const double2 v = __ldg(cp + k);
            c[2 * k] = (R)v.x;
            c[2 * k + 1] = (R)v.y;
        }
    } else {
        const float4* cp = reinterpret_cast<const float4*>(p.coef_aos_f + 24 * (size_t)t);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float4 v = __ldg(cp + k);
            c[4 * k] = (R)v.x;
            c[4 * k + 1] = (R)v.y;
            c[4 * k + 2] = (R)v.z;
            c[4 * k + 3] = (R)v.w;
        }
    }
    // Positions; the mixed path works with differences from vertex 0, formed
    // in double, so the float sums below do not cancel large coordinates.
    double P[6][3];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        P[s][0] = __ldg(pos + ids[s]);
        P[s][1] = __ldg(pos + N + ids[s]);
        P[s][2] = __ldg(pos + 2 * N + ids[s]);
    }
    R Q[6][3];
#pragma unroll
    for (int s = 0; s < 6; ++s)
#pragma unroll
        for (int i = 0; i < 3; ++i) Q[s][i] = MIXED ? (R)(P[s][i] - P[0][i]) : (R)P[s][i];
    R rx[3], ry[3], rxx[3], rxy[3], ryy[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        rx[i] = c[0] * Q[0][i] + c[1] * Q[1][i] + c[2] * Q[2][i];
        ry[i] = c[3] * Q[0][i] + c[4] * Q[1][i] + c[5] * Q[2][i];
        R sxx = 0, sxy = 0, syy = 0;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            sxx += c[6 + 3 * s + 0] * Q[s][i];
            sxy += c[6 + 3 * s + 1] * Q[s][i];
            syy += c[6 + 3 * s + 2] * Q[s][i];
        }
        rxx[i] = sxx;
        rxy[i] = sxy;
        ryy[i] = syy;
    }
    Cq<R> q;
    q.rx = {rx[0], rx[1], rx[2]};
    q.ry = {ry[0], ry[1], ry[2]};
    q.rxx = {rxx[0], rxx[1], rxx[2]};
    q.rxy = {rxy[0], rxy[1], rxy[2]};
    q.ryy = {ryy[0], ryy[1], ryy[2]};
    CqGrad<R> g;
    if constexpr (!MIXED) {
        dev::energy_gradient<double>(q, mt, nu, gamma, g);
    } else {
        double sp, bp;
        dev::prefactors<double>(mt, nu, sp, bp);
        const TriMat<float> mf = {(float)mt.abar0, (float)mt.abar1, (float)mt.abar2, (float)mt.bbar0,
                                  (float)mt.bbar1, (float)mt.bbar2, (float)mt.h, (float)mt.mu, (float)mt.area};
        dev::energy_gradient_pref<float>(q, mf, (float)nu, (float)gamma, (float)sp, (float)bp, g);
    }
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const R mxx = c[6 + 3 * s + 0], mxy = c[6 + 3 * s + 1], myy = c[6 + 3 * s + 2];
        R fx = mxx * g.rxx.x + mxy * g.rxy.x + myy * g.ryy.x;
        R fy = mxx * g.rxx.y + mxy * g.rxy.y + myy * g.ryy.y;
        R fz = mxx * g.rxx.z + mxy * g.rxy.z + myy * g.ryy.z;
        if (s < 3) {
            const R dx = c[s], dy = c[3 + s];
            fx += dx * g.rx.x + dy * g.ry.x;
            fy += dx * g.rx.y + dy * g.ry.y;
            fz += dx * g.rx.z + dy * g.ry.z;
        }
        f[3 * s + 0] = -fx;
        f[3 * s + 1] = -fy;
        f[3 * s + 2] = -fz;
    }
}

}  // namespace tridev
}  // namespace msb
