// CPU restatement of MorphoShell's per-step algorithm (orc_* C ABI of
// oracle.h).  TEST INFRASTRUCTURE ONLY: the checker for the GPU path and the
// "port" CPU baseline.  Parity pinned against the reference's own source
// files compiled here (oracle/_ref, see build.py) on the same inputs.
//
// Sequence and formulas follow:
//   calc_surface_derivs.cpp:27-34      cq = D dofs, each row summed in ascending
//                                      column (node id) order
//   calc_deformation_forces.cpp:40-185 dE/dcq per triangle, F = -D^T dE, each
//                                      dof summed in ascending cq-row order
//   calc_energy_densities.cpp:69-77    the energy density differentiated here
//   do_dialling.cpp:36-260             protocols 1-5 and dialling from an ansatz
//   calc_non_deformation_forces.cpp:44-57, impose_constraints.cpp:56-68,
//   is_at_equilibrium.cpp:62-98, advance_dynamics.cpp:58-93
//   calc_a_comps_and_b_comps_and_normals.cpp, calc_curvatures.cpp,
//   calc_angle_deficits.cpp, calc_energies.cpp, calc_strains.cpp,
//   calc_stresses.cpp                  output quantities
// dE/dcq is computed by forward-mode dual numbers on the energy density, not
// from closed forms, so it checks both the reference's expressions and the
// GPU's chain rule independently.
#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"

namespace {

constexpr int K = 15;

struct Dual {
    double v;
    double d[K];
};

inline Dual dconst(double v) {
    Dual r;
    r.v = v;
    for (int k = 0; k < K; ++k) r.d[k] = 0.0;
    return r;
}
inline Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
inline Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
inline Dual operator*(double s, const Dual& a) {
    Dual r;
    r.v = s * a.v;
    for (int k = 0; k < K; ++k) r.d[k] = s * a.d[k];
    return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
inline Dual dsqrt(const Dual& a) {
    Dual r;
    r.v = std::sqrt(a.v);
    const double h = 0.5 / r.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
    return r;
}

// Quadratic form (1-nu) tr(M^2) + nu tr(M)^2 with M = adj(abar) E, E the
// symmetric tensor (e0, e1; e1, e2).  Works for doubles and duals.
template <typename T>
T quad(double ab0, double ab1, double ab2, const T& e0, const T& e1, const T& e2, double nu) {
    T m00 = ab2 * e0 - ab1 * e1;
    T m01 = ab2 * e1 - ab1 * e2;
    T m10 = ab0 * e1 - ab1 * e0;
    T m11 = ab0 * e2 - ab1 * e1;
    T tr = m00 + m11;
    return (1.0 - nu) * (m00 * m00 + 2.0 * (m01 * m10) + m11 * m11) + nu * (tr * tr);
}
inline double operator_mul_fix(double a) { return a; }

struct Tri {
    int v[3];       // vertex ids
    int p[6];       // patch ids
    double c[24];   // coefficients (ms_mesh_desc layout)
    // surface-derivative rows in ascending node id order
    int ord3[3], ord6[6];
};

struct Ctx {
    int N = 0, T = 0;
    std::vector<Tri> tri;
    std::vector<double> ref_pos, mass, area, thick, shear;
    std::vector<uint8_t> fixed, boundary;
    double nu = 0, gamma = 0, rho = 0, hmin = 0, fchar = 0, vchar = 0, fthr = 0, vthr = 0;
    // node -> (t, slot) in ascending t
    std::vector<int> inc_off, inc_ent;
    // state
    std::vector<double> dofs, vel, forces, cq, dE;
    std::vector<double> abar, bbar, a0, b0;  // T x 3 row-major
    std::vector<double> info_a, info_b;
    int ka = 0, kb = 0, protocol = 1, from_ansatz = 0;
    double spacing = 1.0;
};

// dE_t/dcq of one triangle by forward-mode differentiation of
// A_t [W_s + W_b (1 + W_b/(gamma mu h))].
void tri_energy_grad(const Ctx& c, int t, const double* q, double* out, double* ws_out = nullptr,
                     double* wb_out = nullptr) {
    Dual x[K];
    for (int k = 0; k < K; ++k) {
        x[k] = dconst(q[k]);
        x[k].d[k] = 1.0;
    }
    const Dual* Rx[3] = {&x[0], &x[5], &x[10]};
    const Dual* Ry[3] = {&x[1], &x[6], &x[11]};
    const Dual* Rxx[3] = {&x[2], &x[7], &x[12]};
    const Dual* Rxy[3] = {&x[3], &x[8], &x[13]};
    const Dual* Ryy[3] = {&x[4], &x[9], &x[14]};
    auto dot = [](const Dual* const* a, const Dual* const* b) { return (*a[0]) * (*b[0]) + (*a[1]) * (*b[1]) + (*a[2]) * (*b[2]); };
    const Dual a0 = dot(Rx, Rx), a1 = dot(Rx, Ry), a2 = dot(Ry, Ry);
    Dual cr[3] = {(*Rx[1]) * (*Ry[2]) - (*Rx[2]) * (*Ry[1]), (*Rx[2]) * (*Ry[0]) - (*Rx[0]) * (*Ry[2]),
                  (*Rx[0]) * (*Ry[1]) - (*Rx[1]) * (*Ry[0])};
    const Dual cn = dsqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    Dual n[3] = {cr[0] / cn, cr[1] / cn, cr[2] / cn};
    const Dual* pn[3] = {&n[0], &n[1], &n[2]};
    const Dual b0 = -dot(pn, Rxx), b1 = -dot(pn, Rxy), b2 = -dot(pn, Ryy);

    const double ab0 = c.abar[3 * t], ab1 = c.abar[3 * t + 1], ab2 = c.abar[3 * t + 2];
    const double bb0 = c.bbar[3 * t], bb1 = c.bbar[3 * t + 1], bb2 = c.bbar[3 * t + 2];
    const double h = c.thick[t], mu = c.shear[t], nu = c.nu;
    const double det = ab0 * ab2 - ab1 * ab1;
    const double sp = 2.0 * h * mu / ((1.0 - nu) * det * std::sqrt(det));
    const double bp = mu * h * h * h / (6.0 * (1.0 - nu) * det * std::sqrt(det));
    const Dual ws = (0.5 * sp) * quad(ab0, ab1, ab2, a0 - dconst(ab0), a1 - dconst(ab1), a2 - dconst(ab2), nu);
    const Dual wb = (0.5 * bp) * quad(ab0, ab1, ab2, b0 - dconst(bb0), b1 - dconst(bb1), b2 - dconst(bb2), nu);
    const double scale = c.gamma * mu * h;
    const Dual wbs = wb + (1.0 / scale) * (wb * wb);
    const Dual E = c.area[t] * (ws + wbs);
    for (int k = 0; k < K; ++k) out[k] = E.d[k];
    if (ws_out) *ws_out = ws.v;
    if (wb_out) *wb_out = wbs.v;
}

void surface_derivs(Ctx& c) {
    const int N = c.N;
#pragma omp parallel for schedule(static)
    for (int t = 0; t < c.T; ++t) {
        const Tri& tr = c.tri[t];
        double* q = &c.cq[15 * (size_t)t];
        for (int comp = 0; comp < 3; ++comp) {
            const double* X = &c.dofs[(size_t)comp * N];
            double sx = 0, sy = 0, sxx = 0, sxy = 0, syy = 0;
            for (int j = 0; j < 3; ++j) {
                const int v = tr.ord3[j];
                sx += tr.c[v] * X[tr.v[v]];
                sy += tr.c[3 + v] * X[tr.v[v]];
            }
            for (int j = 0; j < 6; ++j) {
                const int s = tr.ord6[j];
                sxx += tr.c[6 + 3 * s] * X[tr.p[s]];
                sxy += tr.c[6 + 3 * s + 1] * X[tr.p[s]];
                syy += tr.c[6 + 3 * s + 2] * X[tr.p[s]];
            }
            q[5 * comp + 0] = sx;
            q[5 * comp + 1] = sy;
            q[5 * comp + 2] = sxx;
            q[5 * comp + 3] = sxy;
            q[5 * comp + 4] = syy;
        }
    }
}

void deformation_forces(Ctx& c) {
#pragma omp parallel for schedule(static)
    for (int t = 0; t < c.T; ++t) tri_energy_grad(c, t, &c.cq[15 * (size_t)t], &c.dE[15 * (size_t)t]);
    const int N = c.N;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < N; ++n) {
        for (int comp = 0; comp < 3; ++comp) {
            double tmp = 0.0;
            for (int k = c.inc_off[n]; k < c.inc_off[n + 1]; ++k) {
                const int e = c.inc_ent[k], t = e / 6, s = e % 6;
                const Tri& tr = c.tri[t];
                const double* de = &c.dE[15 * (size_t)t + 5 * comp];
                if (s < 3) {
                    tmp += (-tr.c[s]) * de[0];
                    tmp += (-tr.c[3 + s]) * de[1];
                }
                tmp += (-tr.c[6 + 3 * s]) * de[2];
                tmp += (-tr.c[6 + 3 * s + 1]) * de[3];
                tmp += (-tr.c[6 + 3 * s + 2]) * de[4];
            }
            c.forces[(size_t)comp * N + n] = tmp;
        }
    }
}

void non_deformation_forces(Ctx& c, double damping, int gd) {
    if (gd) return;
    const int N = c.N;
    const double rhh = c.rho * c.hmin * c.hmin;
    for (int d = 0; d < 3 * N; ++d) c.forces[d] += -damping * c.mass[d % N] * c.vel[d] / rhh;
}

void constraints(Ctx& c) {
    const int N = c.N;
    for (int n = 0; n < N; ++n)
        if (c.fixed[n]) c.forces[n] = c.forces[N + n] = c.forces[2 * (size_t)N + n] = 0.0;
}

int advance(Ctx& c, double dt, double damping, int gd, int64_t* bad_dof, double* bad_force) {
    const int N = c.N;
    const double lim = 50000.0 * c.fchar;
    for (int d = 0; d < 3 * N; ++d)
        if (!(std::fabs(c.forces[d]) < lim)) {
            if (bad_dof) *bad_dof = d;
            if (bad_force) *bad_force = c.forces[d];
            return 3;
        }
    const double rhh = c.rho * c.hmin * c.hmin;
    for (int d = 0; d < 3 * N; ++d) {
        const double m = c.mass[d % N];
        c.vel[d] += (dt / m) * c.forces[d];
        if (gd) c.vel[d] = rhh * c.forces[d] / (damping * m);
        c.dofs[d] += dt * c.vel[d];
    }
    return 0;
}

void lce(double dial, double angle, double lamf, double nu_ot, double* ab) {
    const double lam = (1.0 - dial) * 1.0 + dial * lamf;
    const double cs = std::cos(angle), sn = std::sin(angle);
    const double p = std::pow(lam, -2.0 * nu_ot);
    ab[0] = lam * lam * cs * cs + p * sn * sn;
    ab[1] = (lam * lam - p) * cs * sn;
    ab[2] = p * cs * cs + lam * lam * sn * sn;
}

void dialling(Ctx& c, double dial_in) {
    const double dial = c.from_ansatz ? 1.0 : dial_in;
    for (int t = 0; t < c.T; ++t) {
        const double* A = &c.info_a[(size_t)t * c.ka];
        const double* B = &c.info_b[(size_t)t * c.kb];
        double* ab = &c.abar[3 * (size_t)t];
        double* bb = &c.bbar[3 * (size_t)t];
        const double* a0 = &c.a0[3 * (size_t)t];
        const double* b0 = &c.b0[3 * (size_t)t];
        switch (c.protocol) {
            case 1:
                for (int k = 0; k < 3; ++k) {
                    ab[k] = (1.0 - dial) * a0[k] + dial * A[k];
                    bb[k] = (1.0 - dial) * b0[k] + dial * B[k];
                }
                break;
            case 2:
                for (int k = 0; k < 3; ++k) {
                    if (dial < 0.5) {
                        ab[k] = a0[k];
                        bb[k] = (1.0 - 2 * dial) * b0[k] + 2 * dial * B[k];
                    } else {
                        ab[k] = (1.0 - 2 * (dial - 0.5)) * a0[k] + 2 * (dial - 0.5) * A[k];
                        bb[k] = B[k];
                    }
                }
                break;
            case 3:
                lce(dial, A[0], A[1], A[2], ab);
                bb[0] = bb[1] = bb[2] = 0.0;
                break;
            case 4: {
                const double nu_ot = A[11], angle = A[12];
                const int idx = std::max(0, std::min((int)std::floor(dial / c.spacing), c.ka - 1));
                const double frac = dial / c.spacing - idx;
                const double prev = A[idx];
                const double next = idx + 1 < c.ka ? A[idx + 1] : prev;
                const double lam = (1 - frac) * prev + frac * next;
                const double cs = std::cos(angle), sn = std::sin(angle), p = std::pow(lam, -2.0 * nu_ot);
                ab[0] = lam * lam * cs * cs + p * sn * sn;
                ab[1] = (lam * lam - p) * cs * sn;
                ab[2] = p * cs * cs + lam * lam * sn * sn;
                bb[0] = bb[1] = bb[2] = 0.0;
                break;
            }
            default: {
                const double r = A[0], absK = dial * 2.0, om = 1.0 / (1.0 - 0.25 * r * r * absK);
                ab[0] = om * om;
                ab[1] = 0.0;
                ab[2] = om * om;
                bb[0] = bb[1] = bb[2] = 0.0;
            }
        }
        if (c.from_ansatz)
            for (int k = 0; k < 3; ++k) {
                ab[k] = (1.0 - dial_in) * a0[k] + dial_in * ab[k];
                bb[k] = (1.0 - dial_in) * b0[k] + dial_in * bb[k];
            }
    }
}

// Upper-triangular R of the Householder QR of a 3x2 matrix (column-major
// F = [R_x R_y]), as in calc_curvatures.cpp:70-77.
void qr_R(const double F[3][2], double R[2][2]) {
    double A[3][2];
    std::memcpy(A, F, sizeof(A));
    for (int k = 0; k < 2; ++k) {
        double tail = 0;
        for (int i = k + 1; i < 3; ++i) tail += A[i][k] * A[i][k];
        const double c0 = A[k][k];
        double beta, tau = 0;
        double v[3] = {0, 0, 0};
        if (tail <= 2.2250738585072014e-308) {
            beta = c0;
        } else {
            beta = std::sqrt(c0 * c0 + tail);
            if (c0 >= 0) beta = -beta;
            for (int i = k + 1; i < 3; ++i) v[i] = A[i][k] / (c0 - beta);
            tau = (beta - c0) / beta;
        }
        v[k] = 1.0;
        for (int j = k + 1; j < 2; ++j) {
            double w = 0;
            for (int i = k; i < 3; ++i) w += v[i] * A[i][j];
            for (int i = k; i < 3; ++i) A[i][j] -= tau * v[i] * w;
        }
        A[k][k] = beta;
    }
    R[0][0] = A[0][0];
    R[0][1] = A[0][1];
    R[1][0] = 0.0;
    R[1][1] = A[1][1];
}

void sym_eig3(const double A[3][3], double w[3], double V[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            a[i][j] = i >= j ? A[i][j] : A[j][i];
            V[i][j] = i == j ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 100; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-36 * dg) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double tt = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double cs = 1.0 / std::sqrt(tt * tt + 1.0), sn = tt * cs;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = cs * akp - sn * akq;
                    a[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = cs * apk - sn * aqk;
                    a[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = cs * vkp - sn * vkq;
                    V[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) w[i] = a[i][i];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2 - i; ++j)
            if (w[j] > w[j + 1]) {
                std::swap(w[j], w[j + 1]);
                for (int k = 0; k < 3; ++k) std::swap(V[k][j], V[k][j + 1]);
            }
}

double kahan(const std::vector<double>& v) {
    double sum = 0.0, comp = 0.0;
    for (double x : v) {
        const double y = x - comp;
        const double t = sum + y;
        comp = (t - sum) - y;
        sum = t;
    }
    return sum;
}

}  // namespace

extern "C" {

void orc_set_threads(int n) { omp_set_num_threads(n); }

void* orc_create(int N, int T, const double* ref_pos, const int32_t* patch, const double*, const double* coeffs,
                 const double* mass, const double* area, const double* thick, const double* shear,
                 const uint8_t* fixed, const uint8_t* boundary, const double* scal) {
    Ctx* c = new Ctx();
    c->N = N;
    c->T = T;
    c->tri.resize(T);
    for (int t = 0; t < T; ++t) {
        Tri& tr = c->tri[t];
        for (int s = 0; s < 6; ++s) tr.p[s] = patch[6 * (size_t)t + s];
        for (int v = 0; v < 3; ++v) tr.v[v] = tr.p[v];
        for (int k = 0; k < 24; ++k) tr.c[k] = coeffs[24 * (size_t)t + k];
        for (int j = 0; j < 3; ++j) tr.ord3[j] = j;
        for (int j = 0; j < 6; ++j) tr.ord6[j] = j;
        std::sort(tr.ord3, tr.ord3 + 3, [&](int a, int b) { return tr.v[a] < tr.v[b]; });
        std::sort(tr.ord6, tr.ord6 + 6, [&](int a, int b) { return tr.p[a] < tr.p[b]; });
    }
    c->ref_pos.assign(ref_pos, ref_pos + 3 * (size_t)N);
    c->mass.assign(mass, mass + N);
    c->area.assign(area, area + T);
    c->thick.assign(thick, thick + T);
    c->shear.assign(shear, shear + T);
    c->fixed.assign(fixed, fixed + N);
    c->boundary.assign(N, 0);
    if (boundary) c->boundary.assign(boundary, boundary + N);
    c->nu = scal[0];
    c->gamma = scal[1];
    c->rho = scal[2];
    c->hmin = scal[3];
    c->fchar = scal[4];
    c->vchar = scal[5];
    c->fthr = scal[6];
    c->vthr = scal[7];
    c->inc_off.assign(N + 1, 0);
    for (int t = 0; t < T; ++t)
        for (int s = 0; s < 6; ++s) c->inc_off[c->tri[t].p[s] + 1] += 1;
    for (int n = 0; n < N; ++n) c->inc_off[n + 1] += c->inc_off[n];
    c->inc_ent.resize(6 * (size_t)T);
    std::vector<int> fill(c->inc_off.begin(), c->inc_off.end() - 1);
    for (int t = 0; t < T; ++t)
        for (int s = 0; s < 6; ++s) c->inc_ent[fill[c->tri[t].p[s]]++] = 6 * t + s;
    c->dofs.assign(3 * (size_t)N, 0.0);
    c->vel.assign(3 * (size_t)N, 0.0);
    c->forces.assign(3 * (size_t)N, 0.0);
    c->cq.assign(15 * (size_t)T, 0.0);
    c->dE.assign(15 * (size_t)T, 0.0);
    c->a0.assign(3 * (size_t)T, 0.0);
    c->b0.assign(3 * (size_t)T, 0.0);
    for (int t = 0; t < T; ++t) c->a0[3 * t] = c->a0[3 * t + 2] = 1.0;
    c->abar = c->a0;
    c->bbar = c->b0;
    return c;
}

void orc_destroy(void* p) { delete static_cast<Ctx*>(p); }

int orc_set_programmed(void* p, int protocol, const double* ai, int ka, const double* bi, int kb, double spacing,
                       int from_ansatz) {
    Ctx& c = *static_cast<Ctx*>(p);
    c.protocol = protocol;
    c.ka = ka;
    c.kb = kb;
    c.info_a.assign(ai, ai + (size_t)c.T * ka);
    c.info_b.assign(bi, bi + (size_t)c.T * kb);
    c.spacing = spacing;
    c.from_ansatz = from_ansatz;
    return 0;
}

void orc_set_zero_dial_state(void* p, const double* a0, const double* b0) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int t = 0; t < c.T; ++t)
        for (int k = 0; k < 3; ++k) {
            c.a0[3 * t + k] = a0 ? a0[3 * t + k] : (k == 1 ? 0.0 : 1.0);
            c.b0[3 * t + k] = b0 ? b0[3 * t + k] : 0.0;
        }
}

void orc_set_state(void* p, const double* dofs, const double* vel) {
    Ctx& c = *static_cast<Ctx*>(p);
    std::memcpy(c.dofs.data(), dofs, sizeof(double) * 3 * c.N);
    if (vel) std::memcpy(c.vel.data(), vel, sizeof(double) * 3 * c.N);
    else std::fill(c.vel.begin(), c.vel.end(), 0.0);
}

void orc_get_state(void* p, double* dofs, double* vel) {
    Ctx& c = *static_cast<Ctx*>(p);
    if (dofs) std::memcpy(dofs, c.dofs.data(), sizeof(double) * 3 * c.N);
    if (vel) std::memcpy(vel, c.vel.data(), sizeof(double) * 3 * c.N);
}

void orc_get_forces(void* p, double* f) {
    Ctx& c = *static_cast<Ctx*>(p);
    std::memcpy(f, c.forces.data(), sizeof(double) * 3 * c.N);
}

void orc_do_dialling(void* p, double dial) { dialling(*static_cast<Ctx*>(p), dial); }

void orc_get_programmed(void* p, double* abar, double* bbar) {
    Ctx& c = *static_cast<Ctx*>(p);
    if (abar) std::memcpy(abar, c.abar.data(), sizeof(double) * 3 * c.T);
    if (bbar) std::memcpy(bbar, c.bbar.data(), sizeof(double) * 3 * c.T);
}

void orc_surface_derivs(void* p, double* cq) {
    Ctx& c = *static_cast<Ctx*>(p);
    surface_derivs(c);
    if (cq) std::memcpy(cq, c.cq.data(), sizeof(double) * 15 * c.T);
}

void orc_a_b_normals(void* p, double* a, double* b, double* n) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int t = 0; t < c.T; ++t) {
        const double* q = &c.cq[15 * (size_t)t];
        const double rx[3] = {q[0], q[5], q[10]}, ry[3] = {q[1], q[6], q[11]};
        const double rxx[3] = {q[2], q[7], q[12]}, rxy[3] = {q[3], q[8], q[13]}, ryy[3] = {q[4], q[9], q[14]};
        a[3 * t] = rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2];
        a[3 * t + 1] = rx[0] * ry[0] + rx[1] * ry[1] + rx[2] * ry[2];
        a[3 * t + 2] = ry[0] * ry[0] + ry[1] * ry[1] + ry[2] * ry[2];
        double cr[3] = {rx[1] * ry[2] - rx[2] * ry[1], rx[2] * ry[0] - rx[0] * ry[2], rx[0] * ry[1] - rx[1] * ry[0]};
        const double nn = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        for (int k = 0; k < 3; ++k) n[3 * t + k] = cr[k] / nn;
        b[3 * t] = -(n[3 * t] * rxx[0] + n[3 * t + 1] * rxx[1] + n[3 * t + 2] * rxx[2]);
        b[3 * t + 1] = -(n[3 * t] * rxy[0] + n[3 * t + 1] * rxy[1] + n[3 * t + 2] * rxy[2]);
        b[3 * t + 2] = -(n[3 * t] * ryy[0] + n[3 * t + 1] * ryy[1] + n[3 * t + 2] * ryy[2]);
    }
}

void orc_deformation_forces(void* p, double* f, double* dE) {
    Ctx& c = *static_cast<Ctx*>(p);
    deformation_forces(c);
    if (f) std::memcpy(f, c.forces.data(), sizeof(double) * 3 * c.N);
    if (dE) std::memcpy(dE, c.dE.data(), sizeof(double) * 15 * c.T);
}

void orc_non_deformation_forces(void* p, double damping, int gd) {
    non_deformation_forces(*static_cast<Ctx*>(p), damping, gd);
}

void orc_impose_constraints(void* p) { constraints(*static_cast<Ctx*>(p)); }

int orc_is_at_equilibrium(void* p, double* out4) {
    Ctx& c = *static_cast<Ctx*>(p);
    const int N = c.N;
    double mf = -1, mv = -1;
    int nf = 0, nv = 0;
    for (int n = 0; n < N; ++n) {
        const double fx = c.forces[n], fy = c.forces[N + n], fz = c.forces[2 * (size_t)N + n];
        const double vx = c.vel[n], vy = c.vel[N + n], vz = c.vel[2 * (size_t)N + n];
        const double f = std::sqrt(fx * fx + fy * fy + fz * fz), v = std::sqrt(vx * vx + vy * vy + vz * vz);
        if (f > mf) { mf = f; nf = n; }
        if (v > mv) { mv = v; nv = n; }
    }
    if (out4) {
        out4[0] = mf;
        out4[1] = mv;
        out4[2] = nf;
        out4[3] = nv;
    }
    return (mf / c.fchar < c.fthr && mv / c.vchar < c.vthr) ? 1 : 0;
}

int orc_advance_dynamics(void* p, double dt, double damping, int gd, int64_t* bad_dof, double* bad_force) {
    return advance(*static_cast<Ctx*>(p), dt, damping, gd, bad_dof, bad_force);
}

int orc_step_n(void* p, int n, const double* dials, double dt, double damping, int gd, int* done) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int i = 0; i < n; ++i) {
        if (done) *done = i;
        surface_derivs(c);
        if (dials) dialling(c, dials[i]);
        deformation_forces(c);
        non_deformation_forces(c, damping, gd);
        constraints(c);
        if (advance(c, dt, damping, gd, nullptr, nullptr) != 0) return 3;
    }
    if (done) *done = n;
    return 0;
}

void orc_output_quantities(void* p, double* curv, double* edens, double* strains, double* stresses,
                           double* deficits, double* energies) {
    Ctx& c = *static_cast<Ctx*>(p);
    const int T = c.T, N = c.N;
    surface_derivs(c);
    std::vector<double> a(3 * (size_t)T), b(3 * (size_t)T), nrm(3 * (size_t)T), es(T), eb(T);
    orc_a_b_normals(p, a.data(), b.data(), nrm.data());
    for (int t = 0; t < T; ++t) {
        const double* q = &c.cq[15 * (size_t)t];
        double g[15], ws, wb;
        tri_energy_grad(c, t, q, g, &ws, &wb);
        es[t] = c.area[t] * ws;
        eb[t] = c.area[t] * wb;
        if (edens) {
            edens[2 * t] = ws;
            edens[2 * t + 1] = wb;
        }
        const double F[3][2] = {{q[0], q[1]}, {q[5], q[6]}, {q[10], q[11]}};
        if (curv) {
            double R[2][2];
            qr_R(F, R);
            const double det = R[0][0] * R[1][1];
            const double iR[2][2] = {{R[1][1] / det, -R[0][1] / det}, {0.0, R[0][0] / det}};
            const double B[2][2] = {{b[3 * t], b[3 * t + 1]}, {b[3 * t + 1], b[3 * t + 2]}};
            double S[2][2] = {{0, 0}, {0, 0}};  // iR^T B iR
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 2; ++j)
                    for (int k = 0; k < 2; ++k)
                        for (int l = 0; l < 2; ++l) S[i][j] += iR[k][i] * B[k][l] * iR[l][j];
            curv[2 * t] = S[0][0] * S[1][1] - S[0][1] * S[1][0];
            curv[2 * t + 1] = 0.5 * (S[0][0] + S[1][1]);
        }
        if (strains) {
            // 0.5 P^T (a - abar) P with P = (F^T F)^-1 F^T; strain = sqrt(tr(E^T E)/2)
            const double A[2][2] = {{a[3 * t], a[3 * t + 1]}, {a[3 * t + 1], a[3 * t + 2]}};
            const double dA = A[0][0] * A[1][1] - A[0][1] * A[1][0];
            const double Ai[2][2] = {{A[1][1] / dA, -A[0][1] / dA}, {-A[1][0] / dA, A[0][0] / dA}};
            double P[2][3];
            for (int i = 0; i < 2; ++i)
                for (int j = 0; j < 3; ++j) P[i][j] = Ai[i][0] * F[j][0] + Ai[i][1] * F[j][1];
            const double D[2][2] = {{A[0][0] - c.abar[3 * t], A[0][1] - c.abar[3 * t + 1]},
                                    {A[1][0] - c.abar[3 * t + 1], A[1][1] - c.abar[3 * t + 2]}};
            double Es[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double s = 0;
                    for (int k = 0; k < 2; ++k)
                        for (int l = 0; l < 2; ++l) s += P[k][i] * D[k][l] * P[l][j];
                    Es[i][j] = 0.5 * s;
                }
            double tr = 0;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) tr += Es[i][j] * Es[i][j];
            strains[t] = std::sqrt(0.5 * tr);
        }
        if (stresses) {
            const double rx[3] = {q[0], q[5], q[10]}, ry[3] = {q[1], q[6], q[11]};
            const double gx[3] = {g[0], g[5], g[10]}, gy[3] = {g[1], g[6], g[11]};
            double cr[3] = {rx[1] * ry[2] - rx[2] * ry[1], rx[2] * ry[0] - rx[0] * ry[2], rx[0] * ry[1] - rx[1] * ry[0]};
            const double J = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            double S[3][3], w[3], V[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) S[i][j] = (gx[i] * rx[j] + gy[i] * ry[j]) / J;
            sym_eig3(S, w, V);
            int im = 0;
            for (int j = 0; j < 3; ++j)
                if (std::fabs(w[im]) > std::fabs(w[j])) im = j;
            const int i1 = (1 + im) % 3, i2 = (2 + im) % 3;
            double* o = stresses + 8 * (size_t)t;
            o[0] = w[i1];
            for (int k = 0; k < 3; ++k) o[1 + k] = V[k][i1];
            o[4] = w[i2];
            for (int k = 0; k < 3; ++k) o[5 + k] = V[k][i2];
        }
    }
    if (deficits) {
        const double pi = 3.14159265358979323846;
        for (int n = 0; n < N; ++n) deficits[n] = c.boundary[n] ? pi : 2.0 * pi;
        for (int t = 0; t < T; ++t) {
            double v[3][3];
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) v[j][k] = c.dofs[(size_t)k * N + c.tri[t].v[j]];
            double s0[3], s1[3], s2[3];
            for (int k = 0; k < 3; ++k) {
                s0[k] = v[1][k] - v[0][k];
                s1[k] = v[2][k] - v[1][k];
                s2[k] = -s1[k] - s0[k];
            }
            auto nr = [](const double* x) { return std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]); };
            auto dt = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
            const double l0 = nr(s0), l1 = nr(s1), l2 = nr(s2);
            deficits[c.tri[t].v[0]] += -std::acos(-dt(s2, s0) / (l2 * l0));
            deficits[c.tri[t].v[1]] += -std::acos(-dt(s0, s1) / (l0 * l1));
            deficits[c.tri[t].v[2]] += -std::acos(-dt(s1, s2) / (l1 * l2));
        }
    }
    if (energies) {
        std::vector<double> ke(N);
        for (int n = 0; n < N; ++n) {
            const double vx = c.vel[n], vy = c.vel[N + n], vz = c.vel[2 * (size_t)N + n];
            ke[n] = 0.5 * c.mass[n] * (vx * vx + vy * vy + vz * vz);
        }
        energies[0] = kahan(es);
        energies[1] = kahan(eb);
        energies[2] = kahan(ke);
    }
}

}  // extern "C"
