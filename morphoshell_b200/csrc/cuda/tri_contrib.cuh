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

// One triangle's 18 contributions into its contrib_stride<MIXED>() staging
// slots (zero padding where the layout has it).
template <bool MIXED>
__device__ __forceinline__ void stage_contrib(typename Real<MIXED>::T* __restrict__ dst,
                                              const typename Real<MIXED>::T (&f)[18]) {
    using R = typename Real<MIXED>::T;
    constexpr int S = contrib_slot<MIXED>();
#pragma unroll
    for (int s = 0; s < 6; ++s) {
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[S * s + c] = f[3 * s + c];
        if constexpr (S == 4) dst[S * s + 3] = R(0);
    }
}

// Material of one triangle with thickness h and shear modulus mu: h, mu and
// their stretch / bend coefficients (the divisions of dev::material_coefs).
__device__ __forceinline__ void set_material(double h, double mu, double nu, double gamma, TriMat<double>& mt) {
    mt.h = h;
    mt.mu = mu;
    dev::material_coefs(h, mu, nu, gamma, mt.ks, mt.kb, mt.igmh);
}

// Material of triangle t: the uniform material's coefficients formed on the
// host, or the triangle's own thickness and shear modulus.
__device__ __forceinline__ void tri_material(const DevMesh& m, int t, TriMat<double>& mt) {
    if (m.uniform_hmu) {
        mt.h = m.h_uniform;
        mt.mu = m.mu_uniform;
        mt.ks = m.ks_uniform;
        mt.kb = m.kb_uniform;
        mt.igmh = m.igmh_uniform;
    } else {
        set_material(__ldg(m.thick + t), __ldg(m.shear + t), m.nu, m.gamma, mt);
    }
}

// Protocol-3 programmed metric (do_dialling.cpp:112-123) from the director
// trigonometry cos^2, sin^2, cos sin and l2 = lambda^2, pp = lambda^(-2 nu_ot);
// bbar = 0.
// The roundings are spelled out (fma, then products) so that every kernel
// that inlines this gets the same bits whatever the compiler would contract.
__device__ __forceinline__ void lce_metric(double c2, double s2, double cs, double l2, double pp,
                                           TriMat<double>& mt) {
    mt.abar0 = __fma_rn(l2, c2, __dmul_rn(pp, s2));
    mt.abar1 = __dmul_rn(__dsub_rn(l2, pp), cs);
    mt.abar2 = __fma_rn(pp, c2, __dmul_rn(l2, s2));
    mt.bbar0 = mt.bbar1 = mt.bbar2 = 0.0;
}

// Contributions of one triangle to its six patch nodes, in the precision of
// the path (double, or float for the mixed path), from its gathered patch
// positions P, its 24 derivative weights c (d/dx, d/dy of the 3 vertices;
// xx, xy, yy weights of the 6 patch nodes) and its material and programmed
// tensors mt.
template <bool MIXED>
__device__ __forceinline__ void tri_forces(const double (&P)[6][3], const typename Real<MIXED>::T (&c)[24],
                                           const TriMat<double>& mt, double nu,
                                           typename Real<MIXED>::T (&f)[18]) {
    using R = typename Real<MIXED>::T;
    Cq<R> q;
    CqGrad<R> g;
    if constexpr (!MIXED) {
        double rx[3], ry[3], rxx[3], rxy[3], ryy[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rx[i] = c[0] * P[0][i] + c[1] * P[1][i] + c[2] * P[2][i];
            ry[i] = c[3] * P[0][i] + c[4] * P[1][i] + c[5] * P[2][i];
            double sxx = 0, sxy = 0, syy = 0;
#pragma unroll
            for (int s = 0; s < 6; ++s) {
                sxx += c[6 + 3 * s + 0] * P[s][i];
                sxy += c[6 + 3 * s + 1] * P[s][i];
                syy += c[6 + 3 * s + 2] * P[s][i];
            }
            rxx[i] = sxx;
            rxy[i] = sxy;
            ryy[i] = syy;
        }
        q.rx = {rx[0], rx[1], rx[2]};
        q.ry = {ry[0], ry[1], ry[2]};
        q.rxx = {rxx[0], rxx[1], rxx[2]};
        q.rxy = {rxy[0], rxy[1], rxy[2]};
        q.ryy = {ryy[0], ryy[1], ryy[2]};
        dev::energy_gradient<double>(q, mt, nu, g);
    } else {
        // Positions relative to vertex 0, formed in double.  The first
        // derivatives and the metric a (hence the strain a - abar) are
        // accumulated in double from the float weights: a is close to abar,
        // so a float a - abar would be mostly rounding noise that changes
        // from state to state, while the rounding of the weights only
        // perturbs the reference triangle by a fixed ~1e-7.  The second
        // derivatives and everything after the strain are float.
        const double dd[6] = {c[0], c[1], c[2], c[3], c[4], c[5]};
        const float* mw = c + 6;
        double Q[6][3];
#pragma unroll
        for (int s = 1; s < 6; ++s)
#pragma unroll
            for (int i = 0; i < 3; ++i) Q[s][i] = P[s][i] - P[0][i];
        double rx[3], ry[3];
        float rxx[3], rxy[3], ryy[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            rx[i] = dd[1] * Q[1][i] + dd[2] * Q[2][i];
            ry[i] = dd[4] * Q[1][i] + dd[5] * Q[2][i];
            float sxx = 0.f, sxy = 0.f, syy = 0.f;
#pragma unroll
            for (int s = 1; s < 6; ++s) {
                const float qf = (float)Q[s][i];
                sxx += mw[3 * s + 0] * qf;
                sxy += mw[3 * s + 1] * qf;
                syy += mw[3 * s + 2] * qf;
            }
            rxx[i] = sxx;
            rxy[i] = sxy;
            ryy[i] = syy;
        }
        const double a0 = rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2];
        const double a1 = rx[0] * ry[0] + rx[1] * ry[1] + rx[2] * ry[2];
        const double a2 = ry[0] * ry[0] + ry[1] * ry[1] + ry[2] * ry[2];
        q.rx = {(float)rx[0], (float)rx[1], (float)rx[2]};
        q.ry = {(float)ry[0], (float)ry[1], (float)ry[2]};
        q.rxx = {rxx[0], rxx[1], rxx[2]};
        q.rxy = {rxy[0], rxy[1], rxy[2]};
        q.ryy = {ryy[0], ryy[1], ryy[2]};
        double sp, bp;
        dev::prefactors<double>(mt, sp, bp);
        const TriMat<float> mf = {(float)mt.abar0, (float)mt.abar1, (float)mt.abar2, (float)mt.bbar0,
                                  (float)mt.bbar1, (float)mt.bbar2, (float)mt.h,    (float)mt.mu,
                                  (float)mt.area,  (float)mt.ks,    (float)mt.kb,    (float)mt.igmh};
        dev::energy_gradient_strain<float>(q, mf, (float)nu, (float)sp, (float)bp,
                                           (float)(a0 - mt.abar0), (float)(a1 - mt.abar1), (float)(a2 - mt.abar2), g);
    }
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        // Second-derivative part: sum_k m_k (ab_k n) = (sum_k m_k ab_k) n.
        const R beta = c[6 + 3 * s + 0] * g.ab[0] + c[6 + 3 * s + 1] * g.ab[1] + c[6 + 3 * s + 2] * g.ab[2];
        R fx = beta * g.n.x;
        R fy = beta * g.n.y;
        R fz = beta * g.n.z;
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


// Contributions of triangle t read from the per-triangle (AoS) tables; mt
// holds the triangle's material (h, mu and their coefficients).
// With DIAL_LCE the programmed metric is protocol 3 at (dial, lam = lambda,
// pw = lambda^(-2 nu_ot)) over the director trigonometry in p.tri_aux;
// otherwise it is read from m.abar / m.bbar.
template <int DIAL, bool MIXED>
__device__ __forceinline__ void tri_contrib(const DevMesh& m, const ClusterPlan& p, const double* __restrict__ pos,
                                            int t, const int (&ids)[6], double dial, double lam, double pw,
                                            typename Real<MIXED>::T (&f)[18], double nu, TriMat<double> mt) {
    using R = typename Real<MIXED>::T;
    const int N = m.N;
    if (DIAL == DIAL_LCE) {
        const double2* ap = reinterpret_cast<const double2*>(p.tri_aux + t);
        const double2 a01 = __ldg(ap), a23 = __ldg(ap + 1);
        mt.area = a01.x;
        double l2 = __dmul_rn(lam, lam), pp = pw;
        if (!p.lce_uniform) {
            const double2 ln = __ldg(p.lce_ln + t);
            const double lt = (1.0 - dial) * 1.0 + dial * ln.x;
            l2 = __dmul_rn(lt, lt);
            pp = pow(lt, -2.0 * ln.y);
        }
        lce_metric(a01.y, a23.x, a23.y, l2, pp, mt);
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
            c[2 * k] = v.x;
            c[2 * k + 1] = v.y;
        }
    } else {
        const float4* cp = reinterpret_cast<const float4*>(p.coef_aos_f + 24 * (size_t)t);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float4 v = __ldg(cp + k);
            c[4 * k] = v.x;
            c[4 * k + 1] = v.y;
            c[4 * k + 2] = v.z;
            c[4 * k + 3] = v.w;
        }
    }
    double P[6][3];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        P[s][0] = __ldg(pos + ids[s]);
        P[s][1] = __ldg(pos + N + ids[s]);
        P[s][2] = __ldg(pos + 2 * N + ids[s]);
    }
    tri_forces<MIXED>(P, c, mt, nu, f);
}

}  // namespace tridev
}  // namespace msb
