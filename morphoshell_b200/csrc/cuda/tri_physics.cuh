// Per-triangle shell physics, written as the chain rule through the surface
// metric a, the unit normal n and the curvature tensor b.
//
// Energy per triangle (source_files/calc_energy_densities.cpp:69-77, the
// handbook's Koiter-type density with bend stiffening):
//
//   E_t = A_t [ W_s + W_b (1 + W_b / (gamma mu h)) ]
//   W_s = sp/2 [ (1-nu) tr(M^2) + nu tr(M)^2 ],  M = adj(abar) (a - abar)
//   W_b = bp/2 [ (1-nu) tr(N^2) + nu tr(N)^2 ],  N = adj(abar) (b - bbar)
//   sp  = 2 h mu / ((1-nu) det(abar)^{3/2}),  bp = mu h^3 / (6 (1-nu) det(abar)^{3/2})
//
// with a_ab = R_a . R_b, n = R_x x R_y / |R_x x R_y|, b_ab = -n . R_ab, and
// R_x ... R_yy the 15 "continuum quantities" of the triangle.  The reference
// (calc_deformation_forces.cpp:93-171) evaluates dE_t/d(cq) from expanded
// Mathematica closed forms; here the same derivatives come from
//
//   dE/dR_x = A (2 s0 R_x + s1 R_y) + A (R_y x g),   s_k = dW_s/da_k
//   dE/dR_y = A (s1 R_x + 2 s2 R_y) + A (g x R_x)
//   dE/dR_ab = -A beta_ab n,                          beta_k = dW_b'/db_k
//   g = -(G - (n.G) n) / |R_x x R_y|,                 G = sum_k beta_k R_k
//
// (a1 and b1 each appear twice in their symmetric tensors, so s1 and beta_1
// are the derivatives with respect to the single off-diagonal component).
// About 400 FP64 operations per triangle instead of ~3.5k.
#pragma once

#include <cuda_runtime.h>

namespace msb {
namespace dev {

template <typename R>
struct V3 {
    R x, y, z;
};

template <typename R>
__device__ __forceinline__ V3<R> cross(const V3<R>& a, const V3<R>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R>
__device__ __forceinline__ R dot(const V3<R>& a, const V3<R>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

__device__ __forceinline__ double rsqrt_r(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_r(float x) { return rsqrtf(x); }

// The 15 continuum quantities of one triangle.
template <typename R>
struct Cq {
    V3<R> rx, ry, rxx, rxy, ryy;
};

// Material and programmed-tensor inputs of one triangle.  ks, kb and igmh
// are the material's stretch and bend coefficients and the bend-stiffening
// scale (material_coefs), formed once per material rather than per triangle
// so that the per-triangle chain carries no division.
template <typename R>
struct TriMat {
    R abar0, abar1, abar2;
    R bbar0, bbar1, bbar2;
    R h, mu, area;
    R ks, kb, igmh;
};

// ks = 2 h mu / (1 - nu), kb = mu h^3 / (6 (1 - nu)), igmh = 1 / (gamma mu h).
// Host and device evaluate the same expressions (products and correctly
// rounded divisions only), so a constant formed on the host for a uniform
// material has the bits the device forms per triangle otherwise.
template <typename R>
__host__ __device__ __forceinline__ void material_coefs(R h, R mu, R nu, R gamma, R& ks, R& kb, R& igmh) {
    const R omn = R(1) - nu;
    ks = R(2) * h * mu / omn;
    kb = mu * h * h * h / (R(6) * omn);
    igmh = R(1) / (gamma * mu * h);
}

// dE_t / d(cq), grouped as the 5 vector derivatives.
template <typename R>
struct CqGrad {
    V3<R> rx, ry, rxx, rxy, ryy;
    // The three second-derivative gradients are multiples of the unit
    // normal: dE/dR_ab = ab[k] n (k = xx, xy, yy).
    R ab[3];
    V3<R> n;
};

// Quadratic-form helper: for symmetric D = [[d0, d1], [d1, d2]] and
// adj = adj(abar), returns W = (1-nu) tr(M^2) + nu tr(M)^2 with M = adj D, and
// its derivatives dW/dd0, dW/dd1 (single off-diagonal variable), dW/dd2,
// all without the 1/2 prefactor (so the energy density is pref/2 * W and its
// derivatives are pref * q).
template <typename R>
__device__ __forceinline__ R quad_form(R abar0, R abar1, R abar2, R d0, R d1, R d2, R nu, R& q0, R& q1, R& q2) {
    const R m00 = abar2 * d0 - abar1 * d1;
    const R m01 = abar2 * d1 - abar1 * d2;
    const R m10 = abar0 * d1 - abar1 * d0;
    const R m11 = abar0 * d2 - abar1 * d1;
    const R tr = m00 + m11;
    const R omn = R(1) - nu;
    const R w = omn * (m00 * m00 + R(2) * m01 * m10 + m11 * m11) + nu * tr * tr;
    // S = (1-nu) M + nu tr I;  Q = S adj (symmetric); dW/dD = 2 Q.
    const R s00 = omn * m00 + nu * tr;
    const R s01 = omn * m01;
    const R s10 = omn * m10;
    const R s11 = omn * m11 + nu * tr;
    q0 = s00 * abar2 - s01 * abar1;
    const R qa = s01 * abar0 - s00 * abar1;
    const R qb = s10 * abar2 - s11 * abar1;
    q1 = qa + qb;
    q2 = s11 * abar0 - s10 * abar1;
    return w;
}

// Stretch and bend prefactors sp, bp of one triangle (they hold the metric
// inverse through det(abar)^(-3/2), formed as the cube of one reciprocal
// square root: a few ulp, and no division on the chain).
template <typename R>
__device__ __forceinline__ void prefactors(const TriMat<R>& m, R& sp, R& bp) {
    const R det = m.abar0 * m.abar2 - m.abar1 * m.abar1;
    const R r = rsqrt_r(det);
    const R det_m32 = r * r * r;
    sp = m.ks * det_m32;
    bp = m.kb * det_m32;
}

template <typename R>
__device__ __forceinline__ void energy_gradient_pref(const Cq<R>& c, const TriMat<R>& m, R nu, R sp, R bp,
                                                     CqGrad<R>& g, R* w_stretch = nullptr, R* w_bend = nullptr);
template <typename R>
__device__ __forceinline__ void energy_gradient_strain(const Cq<R>& c, const TriMat<R>& m, R nu, R sp, R bp, R d0,
                                                       R d1, R d2, CqGrad<R>& g, R* w_stretch = nullptr,
                                                       R* w_bend = nullptr);

// Energy gradient of one triangle.  Also returns the stretch and bend
// (stiffened) energy densities, used by the energy reductions.
template <typename R>
__device__ __forceinline__ void energy_gradient(const Cq<R>& c, const TriMat<R>& m, R nu, CqGrad<R>& g,
                                                R* w_stretch = nullptr, R* w_bend = nullptr) {
    R sp, bp;
    prefactors(m, sp, bp);
    energy_gradient_pref(c, m, nu, sp, bp, g, w_stretch, w_bend);
}

// The same with the prefactors given.
template <typename R>
__device__ __forceinline__ void energy_gradient_pref(const Cq<R>& c, const TriMat<R>& m, R nu, R sp, R bp,
                                                     CqGrad<R>& g, R* w_stretch, R* w_bend) {
    const R a0 = dot(c.rx, c.rx), a1 = dot(c.rx, c.ry), a2 = dot(c.ry, c.ry);
    energy_gradient_strain(c, m, nu, sp, bp, a0 - m.abar0, a1 - m.abar1, a2 - m.abar2, g, w_stretch, w_bend);
}

// The same with the stretch strain d = a - abar given.  The mixed-precision
// path forms d in double (a ~ 1 while d is small, so a float a - abar would
// lose most of d's digits) and the prefactors in double, and runs the rest in
// float.
template <typename R>
__device__ __forceinline__ void energy_gradient_strain(const Cq<R>& c, const TriMat<R>& m, R nu, R sp, R bp, R d0,
                                                       R d1, R d2, CqGrad<R>& g, R* w_stretch, R* w_bend) {
    // Stretch.
    R qs0, qs1, qs2;
    const R ws = quad_form(m.abar0, m.abar1, m.abar2, d0, d1, d2, nu, qs0, qs1, qs2);
    // dW_s/da_k = sp * q_k.
    const R s0 = sp * qs0, s1 = sp * qs1, s2 = sp * qs2;

    // Bend.
    const V3<R> cn = cross(c.rx, c.ry);
    const R inv_c = rsqrt_r(dot(cn, cn));
    const V3<R> n = {cn.x * inv_c, cn.y * inv_c, cn.z * inv_c};
    const R b0 = -dot(n, c.rxx), b1 = -dot(n, c.rxy), b2 = -dot(n, c.ryy);
    R qb0, qb1, qb2;
    const R wb_raw = quad_form(m.abar0, m.abar1, m.abar2, b0 - m.bbar0, b1 - m.bbar1, b2 - m.bbar2, nu, qb0, qb1, qb2);
    const R wb = R(0.5) * bp * wb_raw;
    const R fac = R(1) + R(2) * wb * m.igmh;
    const R bpf = bp * fac;
    const R be0 = bpf * qb0, be1 = bpf * qb1, be2 = bpf * qb2;

    // G = sum beta_k R_k ; g = -(G - (n.G) n) / |c|
    const V3<R> G = {be0 * c.rxx.x + be1 * c.rxy.x + be2 * c.ryy.x, be0 * c.rxx.y + be1 * c.rxy.y + be2 * c.ryy.y,
                     be0 * c.rxx.z + be1 * c.rxy.z + be2 * c.ryy.z};
    const R nG = dot(n, G);
    const V3<R> gv = {(nG * n.x - G.x) * inv_c, (nG * n.y - G.y) * inv_c, (nG * n.z - G.z) * inv_c};
    const V3<R> ryxg = cross(c.ry, gv);
    const V3<R> gxrx = cross(gv, c.rx);
    const R A = m.area;
    const R two = R(2);
    g.rx = {A * (two * s0 * c.rx.x + s1 * c.ry.x + ryxg.x), A * (two * s0 * c.rx.y + s1 * c.ry.y + ryxg.y),
            A * (two * s0 * c.rx.z + s1 * c.ry.z + ryxg.z)};
    g.ry = {A * (s1 * c.rx.x + two * s2 * c.ry.x + gxrx.x), A * (s1 * c.rx.y + two * s2 * c.ry.y + gxrx.y),
            A * (s1 * c.rx.z + two * s2 * c.ry.z + gxrx.z)};
    const R Ab0 = -A * be0, Ab1 = -A * be1, Ab2 = -A * be2;
    g.ab[0] = Ab0;
    g.ab[1] = Ab1;
    g.ab[2] = Ab2;
    g.n = n;
    g.rxx = {Ab0 * n.x, Ab0 * n.y, Ab0 * n.z};
    g.rxy = {Ab1 * n.x, Ab1 * n.y, Ab1 * n.z};
    g.ryy = {Ab2 * n.x, Ab2 * n.y, Ab2 * n.z};
    if (w_stretch) *w_stretch = R(0.5) * sp * ws;
    if (w_bend) *w_bend = wb * (R(1) + wb * m.igmh);
}

// LCE metric of dialling protocol 3 (do_dialling.cpp:112-123): lambda along
// the director at `angle`, lambda^(-2 nu_ot) across it.
__device__ __forceinline__ void lce_abar(double dial, double angle, double lam_final, double nu_ot, double& a0,
                                         double& a1, double& a2) {
    const double lam = (1.0 - dial) * 1.0 + dial * lam_final;
    double s, c;
    sincos(angle, &s, &c);
    const double p = pow(lam, -2.0 * nu_ot);
    const double l2 = lam * lam;
    a0 = l2 * c * c + p * s * s;
    a1 = (l2 - p) * c * s;
    a2 = p * c * c + l2 * s * s;
}

}  // namespace dev
}  // namespace msb
