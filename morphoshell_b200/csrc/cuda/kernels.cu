// sm_100a kernels of the force-and-dynamics loop.
//
// Two-kernel fused path (ms_set_step_path 1 and 2; the default on meshes too
// small for the node-tiled one-kernel step of node_tiles.cu): the
// per-triangle kernel (k_tri_aos in cluster.cu, or k_tri_tiles in
// tri_tiles.cu) writes each triangle's 6 per-node force contributions, then
//   k_node_update one thread per node: deterministic gather of its
//                 contributions in ascending triangle order (the transposed
//                 SpMV of calc_deformation_forces.cpp:185), damping
//                 (calc_non_deformation_forces.cpp:44-57), constraints
//                 (impose_constraints.cpp:56-68), the equilibrium maxima
//                 (is_at_equilibrium.cpp:62-84), the force guard and the
//                 symplectic Euler update (advance_dynamics.cpp:58-93).
// No floating-point atomics anywhere: every sum has a fixed order, so runs
// are bitwise reproducible.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <type_traits>

#include "internal.cuh"
#include "step_common.cuh"
#include "tri_physics.cuh"

namespace msb {

using dev::Cq;
using dev::CqGrad;
using dev::TriMat;
using dev::V3;
using namespace stepdev;

namespace {

constexpr int kNodeBlock = 256;

template <typename R>
__device__ __forceinline__ void load_cq_from_patch(const DevMesh& m, const double* __restrict__ pos, int t,
                                                   const int (&ids)[6], Cq<R>& c, R (&coef)[24]) {
    const int T = m.T, N = m.N;
#pragma unroll
    for (int k = 0; k < 24; ++k) coef[k] = (R)__ldg(m.coef + (size_t)k * T + t);
    R P[6][3];
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        P[s][0] = (R)__ldg(pos + ids[s]);
        P[s][1] = (R)__ldg(pos + N + ids[s]);
        P[s][2] = (R)__ldg(pos + 2 * N + ids[s]);
    }
    R rx[3], ry[3], rxx[3], rxy[3], ryy[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        rx[i] = coef[0] * P[0][i] + coef[1] * P[1][i] + coef[2] * P[2][i];
        ry[i] = coef[3] * P[0][i] + coef[4] * P[1][i] + coef[5] * P[2][i];
        R sxx = 0, sxy = 0, syy = 0;
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            sxx += coef[6 + 3 * s + 0] * P[s][i];
            sxy += coef[6 + 3 * s + 1] * P[s][i];
            syy += coef[6 + 3 * s + 2] * P[s][i];
        }
        rxx[i] = sxx;
        rxy[i] = sxy;
        ryy[i] = syy;
    }
    c.rx = {rx[0], rx[1], rx[2]};
    c.ry = {ry[0], ry[1], ry[2]};
    c.rxx = {rxx[0], rxx[1], rxx[2]};
    c.rxy = {rxy[0], rxy[1], rxy[2]};
    c.ryy = {ryy[0], ryy[1], ryy[2]};
}

__device__ __forceinline__ void load_material(const DevMesh& m, int t, TriMat<double>& mt) {
    if (m.uniform_hmu) {
        mt.h = m.h_uniform;
        mt.mu = m.mu_uniform;
        mt.ks = m.ks_uniform;
        mt.kb = m.kb_uniform;
        mt.igmh = m.igmh_uniform;
    } else {
        mt.h = __ldg(m.thick + t);
        mt.mu = __ldg(m.shear + t);
        dev::material_coefs(mt.h, mt.mu, m.nu, m.gamma, mt.ks, mt.kb, mt.igmh);
    }
    mt.area = __ldg(m.area + t);
}

// Force contributions of one triangle on its 6 patch nodes: slot s gets
// -(sum over the triangle's cq rows of D[row, node_s] * dE/dcq[row]).
template <typename R>
__device__ __forceinline__ void slot_forces(const R (&coef)[24], const CqGrad<R>& g, R (&f)[18]) {
#pragma unroll
    for (int s = 0; s < 6; ++s) {
        const R mxx = coef[6 + 3 * s + 0], mxy = coef[6 + 3 * s + 1], myy = coef[6 + 3 * s + 2];
        R fx = mxx * g.rxx.x + mxy * g.rxy.x + myy * g.ryy.x;
        R fy = mxx * g.rxx.y + mxy * g.rxy.y + myy * g.ryy.y;
        R fz = mxx * g.rxx.z + mxy * g.rxy.z + myy * g.ryy.z;
        if (s < 3) {
            const R dx = coef[s], dy = coef[3 + s];
            fx += dx * g.rx.x + dy * g.ry.x;
            fy += dx * g.rx.y + dy * g.ry.y;
            fz += dx * g.rx.z + dy * g.ry.z;
        }
        f[3 * s + 0] = -fx;
        f[3 * s + 1] = -fy;
        f[3 * s + 2] = -fz;
    }
}

// Block-wide max with first-index tie-break, then the last block to finish
// folds the per-block partials in block order.
__device__ __forceinline__ void eq_block_reduce_and_finish(const DevState& s, double fmax, int fnode, double vmax,
                                                           int vnode) {
    const EqPartial r = eq_block_reduce<kNodeBlock>(fmax, fnode, vmax, vnode);
    eq_store_and_fold(s, r, blockIdx.x, gridDim.x, gridDim.x);
}

// Resident blocks the node kernel asks the compiler for: the FP64 gather
// holds more in flight per thread and is best unconstrained (64 registers);
// the mixed one is best at 48 registers, five blocks per SM (measured).
#ifndef MSB_NODE_MINB
#define MSB_NODE_MINB 1
#endif
#ifndef MSB_NODE_MINB_MIXED
#define MSB_NODE_MINB_MIXED 5
#endif
#ifndef MSB_NODE_REVERSE
#define MSB_NODE_REVERSE 1
#endif

template <bool MIXED>
__global__ void __launch_bounds__(kNodeBlock, MIXED ? MSB_NODE_MINB_MIXED : MSB_NODE_MINB)
    k_node_update(const DevMesh m, const DevState s, const StepScalars sc) {
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform: only earlier kernels can make it true
    // Blocks take the nodes from the top down: the per-triangle kernel wrote
    // the contributions of the last (Morton-ordered) triangles last, so
    // those are still in L2 when the highest nodes start; and the lowest
    // nodes, updated last, are the first the next step's triangles read.
    const int nb = MSB_NODE_REVERSE ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x;
    const int n = nb * kNodeBlock + threadIdx.x;
    const int N = m.N;
    double fmax = -1.0, vmax = -1.0;
    int fnode = INT_MAX, vnode = INT_MAX;
    if ((n & ~31) < N) {  // warp-uniform; lanes past N walk padding only
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        if constexpr (MIXED) gather_sell<float>(m, m.contrib_f, n, Fx, Fy, Fz);
        else gather_sell<double>(m, s.contrib, n, Fx, Fy, Fz);
        if (n < N) node_finish(m, s, sc, gstep, n, Fx, Fy, Fz, fmax, fnode, vmax, vnode);
    }
    if (sc.check) eq_block_reduce_and_finish(s, fmax, fnode, vmax, vnode);
}

// ---- one call per reference function ---------------------------------------

__global__ void k_surface_derivs(const DevMesh m, const DevState s, int parity) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    int ids[6];
    for (int k = 0; k < 6; ++k) ids[k] = m.patch[(size_t)k * m.T + t];
    Cq<double> c;
    double coef[24];
    load_cq_from_patch<double>(m, pos_buf(s, parity), t, ids, c, coef);
    double* o = s.cq + (size_t)t * 15;
    o[0] = c.rx.x; o[1] = c.ry.x; o[2] = c.rxx.x; o[3] = c.rxy.x; o[4] = c.ryy.x;
    o[5] = c.rx.y; o[6] = c.ry.y; o[7] = c.rxx.y; o[8] = c.rxy.y; o[9] = c.ryy.y;
    o[10] = c.rx.z; o[11] = c.ry.z; o[12] = c.rxx.z; o[13] = c.rxy.z; o[14] = c.ryy.z;
}

__device__ __forceinline__ void read_cq(const double* q, Cq<double>& c) {
    c.rx = {q[0], q[5], q[10]};
    c.ry = {q[1], q[6], q[11]};
    c.rxx = {q[2], q[7], q[12]};
    c.rxy = {q[3], q[8], q[13]};
    c.ryy = {q[4], q[9], q[14]};
}

__global__ void k_forces_from_cq(const DevMesh m, const DevState s, int write_dE) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    Cq<double> c;
    read_cq(s.cq + (size_t)t * 15, c);
    TriMat<double> mt;
    load_material(m, t, mt);
    mt.abar0 = m.abar[t];
    mt.abar1 = m.abar[(size_t)m.T + t];
    mt.abar2 = m.abar[2 * (size_t)m.T + t];
    mt.bbar0 = m.bbar[t];
    mt.bbar1 = m.bbar[(size_t)m.T + t];
    mt.bbar2 = m.bbar[2 * (size_t)m.T + t];
    CqGrad<double> g;
    dev::energy_gradient<double>(c, mt, m.nu, g);
    if (write_dE) {
        double* o = s.dEdcq + (size_t)t * 15;
        o[0] = g.rx.x; o[1] = g.ry.x; o[2] = g.rxx.x; o[3] = g.rxy.x; o[4] = g.ryy.x;
        o[5] = g.rx.y; o[6] = g.ry.y; o[7] = g.rxx.y; o[8] = g.rxy.y; o[9] = g.ryy.y;
        o[10] = g.rx.z; o[11] = g.ry.z; o[12] = g.rxx.z; o[13] = g.rxy.z; o[14] = g.ryy.z;
    }
    double coef[24];
    for (int k = 0; k < 24; ++k) coef[k] = m.coef[(size_t)k * m.T + t];
    double f[18];
    slot_forces<double>(coef, g, f);
    for (int j = 0; j < 18; ++j) s.contrib[(size_t)t * 18 + j] = f[j];
}

__global__ void k_gather_forces(const DevMesh m, const DevState s) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    double F[3] = {0.0, 0.0, 0.0};
    for (int k = m.inc_off[n]; k < m.inc_off[n + 1]; ++k) {
        const int e = m.inc_ent[k];
        for (int c = 0; c < 3; ++c) F[c] += s.contrib[3 * (size_t)e + c];
    }
    for (int c = 0; c < 3; ++c) s.forces[(size_t)c * m.N + n] = F[c];
}

__global__ void k_damping(const DevMesh m, const DevState s, int parity, double damping, double rho_hh) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const double dm = -damping * m.mass[n] / rho_hh;
    for (int c = 0; c < 3; ++c) s.forces[(size_t)c * m.N + n] += dm * vel_buf(s, parity)[(size_t)c * m.N + n];
}

__global__ void k_constraints(const DevMesh m, const DevState s) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    if (m.fixed[n])
        for (int c = 0; c < 3; ++c) s.forces[(size_t)c * m.N + n] = 0.0;
}

__global__ void __launch_bounds__(kNodeBlock) k_equilibrium(const DevMesh m, const DevState s, int parity) {
    const int n = blockIdx.x * kNodeBlock + threadIdx.x;
    double f = -1.0, v = -1.0;
    int fn = INT_MAX, vn = INT_MAX;
    if (n < m.N) {
        const size_t N = m.N;
        const double Fx = s.forces[n], Fy = s.forces[N + n], Fz = s.forces[2 * N + n];
        const double* vel = vel_buf(s, parity);
        const double vx = vel[n], vy = vel[N + n], vz = vel[2 * N + n];
        f = sqrt(Fx * Fx + Fy * Fy + Fz * Fz);
        v = sqrt(vx * vx + vy * vy + vz * vz);
        fn = vn = n;
    }
    eq_block_reduce_and_finish(s, f, fn, v, vn);
}

__global__ void k_guard(const DevMesh m, const DevState s, double lim) {
    const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= 3LL * m.N) return;
    if (!(fabs(s.forces[d]) < lim)) {
        atomicMin(&s.err->guard_key, (unsigned long long)d);
        atomicExch(&s.err->flag, 3);
    }
}

__global__ void k_advance(const DevMesh m, const DevState s, int parity, double dt, double damping, double rho_hh,
                          int gd) {
    const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= 3LL * m.N) return;
    const double mass = m.mass[d % m.N];
    double* vel = vel_buf(s, parity);
    double* pos = pos_buf(s, parity);
    const double F = s.forces[d];
    double v = vel[d] + (dt / mass) * F;
    if (gd) v = rho_hh * F / (damping * mass);
    vel[d] = v;
    pos[d] = pos[d] + dt * v;
}

// ---- dialling (do_dialling.cpp:36-260) ---------------------------------------

__global__ void k_dialling(const DevMesh m, int protocol, double dial_in, double spacing, int from_ansatz) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    const size_t T = m.T;
    auto IA = [&](int col) { return m.info_a[(size_t)col * T + t]; };
    auto IB = [&](int col) { return m.info_b[(size_t)col * T + t]; };
    const double dial = from_ansatz ? 1.0 : dial_in;
    double ab[3], bb[3];
    double a0[3], b0[3];
    for (int k = 0; k < 3; ++k) {
        a0[k] = m.a0[k * T + t];
        b0[k] = m.b0[k * T + t];
    }
    if (protocol == 1) {
        for (int k = 0; k < 3; ++k) {
            ab[k] = (1.0 - dial) * a0[k] + dial * IA(k);
            bb[k] = (1.0 - dial) * b0[k] + dial * IB(k);
        }
    } else if (protocol == 2) {
        if (dial < 0.5) {
            for (int k = 0; k < 3; ++k) {
                ab[k] = a0[k];
                bb[k] = (1.0 - 2 * dial) * b0[k] + 2 * dial * IB(k);
            }
        } else {
            for (int k = 0; k < 3; ++k) {
                ab[k] = (1.0 - 2 * (dial - 0.5)) * a0[k] + 2 * (dial - 0.5) * IA(k);
                bb[k] = IB(k);
            }
        }
    } else if (protocol == 3) {
        dev::lce_abar(dial, IA(0), IA(1), IA(2), ab[0], ab[1], ab[2]);
        bb[0] = bb[1] = bb[2] = 0.0;
    } else if (protocol == 4) {
        const double nu_ot = IA(11);
        const double angle = IA(12);
        // The reference reads columns idx and idx + 1 unchecked; keep both
        // inside the table (the last checkpoint holds beyond its range).
        const int idx = max(0, min((int)floor(dial / spacing), m.ka - 1));
        const double frac = dial / spacing - idx;
        const double prev = IA(idx);
        const double next = (idx + 1 < m.ka) ? IA(idx + 1) : prev;
        const double lam = (1 - frac) * prev + frac * next;
        double s, c;
        sincos(angle, &s, &c);
        const double p = pow(lam, -2.0 * nu_ot);
        ab[0] = lam * lam * c * c + p * s * s;
        ab[1] = (lam * lam - p) * c * s;
        ab[2] = p * c * c + lam * lam * s * s;
        bb[0] = bb[1] = bb[2] = 0.0;
    } else {  // 5: isotropic swelling
        const double r = IA(0);
        const double absK = dial * 2.0;
        const double omega = 1.0 / (1.0 - 0.25 * r * r * absK);
        ab[0] = omega * omega;
        ab[1] = 0.0;
        ab[2] = omega * omega;
        bb[0] = bb[1] = bb[2] = 0.0;
    }
    if (from_ansatz) {
        for (int k = 0; k < 3; ++k) {
            ab[k] = (1.0 - dial_in) * a0[k] + dial_in * ab[k];
            bb[k] = (1.0 - dial_in) * b0[k] + dial_in * bb[k];
        }
    }
    for (int k = 0; k < 3; ++k) {
        m.abar[k * T + t] = ab[k];
        m.bbar[k * T + t] = bb[k];
    }
}

// ---- output diagnostics -------------------------------------------------------

__global__ void k_a_b_normals(const DevMesh m, const DevState s, double* a, double* b, double* nrm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    Cq<double> c;
    read_cq(s.cq + (size_t)t * 15, c);
    const V3<double> cr = dev::cross(c.rx, c.ry);
    const double inv = 1.0 / sqrt(dev::dot(cr, cr));
    const V3<double> n = {cr.x * inv, cr.y * inv, cr.z * inv};
    a[3 * (size_t)t + 0] = dev::dot(c.rx, c.rx);
    a[3 * (size_t)t + 1] = dev::dot(c.rx, c.ry);
    a[3 * (size_t)t + 2] = dev::dot(c.ry, c.ry);
    nrm[3 * (size_t)t + 0] = n.x;
    nrm[3 * (size_t)t + 1] = n.y;
    nrm[3 * (size_t)t + 2] = n.z;
    b[3 * (size_t)t + 0] = -dev::dot(n, c.rxx);
    b[3 * (size_t)t + 1] = -dev::dot(n, c.rxy);
    b[3 * (size_t)t + 2] = -dev::dot(n, c.ryy);
}

// Symmetric 3x3 eigen-decomposition (cyclic Jacobi), ascending eigenvalues,
// eigenvectors in the columns of V.  Reads the lower triangle, as a
// self-adjoint solver does.
__device__ void sym_eig3(const double (&A)[3][3], double (&w)[3], double (&V)[3][3]) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            a[i][j] = (i >= j) ? A[i][j] : A[j][i];
            V[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-36 * dg) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double tt = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double cs = 1.0 / sqrt(tt * tt + 1.0), sn = tt * cs;
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
                const double tw = w[j];
                w[j] = w[j + 1];
                w[j + 1] = tw;
                for (int k = 0; k < 3; ++k) {
                    const double tv = V[k][j];
                    V[k][j] = V[k][j + 1];
                    V[k][j + 1] = tv;
                }
            }
}

// Per-triangle output quantities: curvatures (Gauss = det b / det a, mean =
// tr(a^-1 b)/2, the invariants of calc_curvatures.cpp's symmetric shape
// operator), energy densities (calc_energy_densities.cpp), strain
// (calc_strains.cpp: sqrt(tr((a^-1 (a - abar))^2) / 8), the RMS principal
// strain of its pseudo-inverse strain tensor), Cauchy stress eigenpairs
// (calc_stresses.cpp: sigma_ij = sum_alpha dE/dR_alpha,i R_alpha,j / sqrt(det a),
// keeping the two eigenpairs other than the smallest-magnitude one), and
// area-weighted energies for the totals of calc_energies.cpp.
__global__ void k_output_tri(const DevMesh m, const DevState s, double* curv, double* edens, double* strain,
                             double* stress, double* tri_energy) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m.T) return;
    const size_t T = m.T;
    Cq<double> c;
    read_cq(s.cq + (size_t)t * 15, c);
    TriMat<double> mt;
    load_material(m, t, mt);
    mt.abar0 = m.abar[t];
    mt.abar1 = m.abar[T + t];
    mt.abar2 = m.abar[2 * T + t];
    mt.bbar0 = m.bbar[t];
    mt.bbar1 = m.bbar[T + t];
    mt.bbar2 = m.bbar[2 * T + t];
    CqGrad<double> g;
    double ws, wb;
    dev::energy_gradient<double>(c, mt, m.nu, g, &ws, &wb);
    const double a0 = dev::dot(c.rx, c.rx), a1 = dev::dot(c.rx, c.ry), a2 = dev::dot(c.ry, c.ry);
    const V3<double> cr = dev::cross(c.rx, c.ry);
    const double cn2 = dev::dot(cr, cr);
    const double inv = 1.0 / sqrt(cn2);
    const V3<double> n = {cr.x * inv, cr.y * inv, cr.z * inv};
    const double b0 = -dev::dot(n, c.rxx), b1 = -dev::dot(n, c.rxy), b2 = -dev::dot(n, c.ryy);
    const double deta = a0 * a2 - a1 * a1;
    if (curv) {
        curv[2 * (size_t)t + 0] = (b0 * b2 - b1 * b1) / deta;
        curv[2 * (size_t)t + 1] = 0.5 * (a2 * b0 - 2.0 * a1 * b1 + a0 * b2) / deta;
    }
    if (edens) {
        edens[2 * (size_t)t + 0] = ws;
        edens[2 * (size_t)t + 1] = wb;
    }
    if (strain) {
        // X = a^-1 (a - abar)
        const double d0 = a0 - mt.abar0, d1 = a1 - mt.abar1, d2 = a2 - mt.abar2;
        const double x00 = (a2 * d0 - a1 * d1) / deta, x01 = (a2 * d1 - a1 * d2) / deta;
        const double x10 = (a0 * d1 - a1 * d0) / deta, x11 = (a0 * d2 - a1 * d1) / deta;
        const double tr2 = x00 * x00 + 2.0 * x01 * x10 + x11 * x11;
        strain[t] = sqrt(0.125 * tr2);
    }
    if (stress) {
        const double invJ = 1.0 / sqrt(cn2);
        const double gx[3] = {g.rx.x, g.rx.y, g.rx.z}, gy[3] = {g.ry.x, g.ry.y, g.ry.z};
        const double rx[3] = {c.rx.x, c.rx.y, c.rx.z}, ry[3] = {c.ry.x, c.ry.y, c.ry.z};
        double S[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) S[i][j] = (gx[i] * rx[j] + gy[i] * ry[j]) * invJ;
        double w[3], V[3][3];
        sym_eig3(S, w, V);
        int imin = 0;
        for (int j = 0; j < 3; ++j)
            if (fabs(w[imin]) > fabs(w[j])) imin = j;
        const int i1 = (1 + imin) % 3, i2 = (2 + imin) % 3;
        double* o = stress + 8 * (size_t)t;
        o[0] = w[i1];
        o[1] = V[0][i1];
        o[2] = V[1][i1];
        o[3] = V[2][i1];
        o[4] = w[i2];
        o[5] = V[0][i2];
        o[6] = V[1][i2];
        o[7] = V[2][i2];
    }
    if (tri_energy) {
        tri_energy[t] = mt.area * ws;
        tri_energy[T + t] = mt.area * wb;
    }
}

// Angle deficits (calc_angle_deficits.cpp:41-78) as a per-node gather over the
// node's incident triangles in ascending triangle order, which is the order
// the reference's serial scatter adds them in.
__global__ void k_angle_deficits(const DevMesh m, const DevState s, int parity, double* out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const double pi = 3.14159265358979323846;
    const double* pos = pos_buf(s, parity);
    const size_t N = m.N, T = m.T;
    double acc = (m.boundary && m.boundary[n]) ? pi : 2.0 * pi;
    for (int k = m.inc_off[n]; k < m.inc_off[n + 1]; ++k) {
        const int e = m.inc_ent[k];
        const int t = e / 6, slot = e % 6;
        if (slot >= 3) continue;
        const int v0 = m.patch[t], v1 = m.patch[T + t], v2 = m.patch[2 * T + t];
        const double p0[3] = {pos[v0], pos[N + v0], pos[2 * N + v0]};
        const double p1[3] = {pos[v1], pos[N + v1], pos[2 * N + v1]};
        const double p2[3] = {pos[v2], pos[N + v2], pos[2 * N + v2]};
        double s0[3], s1[3], s2[3];
        for (int i = 0; i < 3; ++i) {
            s0[i] = p1[i] - p0[i];
            s1[i] = p2[i] - p1[i];
            s2[i] = -s1[i] - s0[i];
        }
        const double l0 = sqrt(s0[0] * s0[0] + s0[1] * s0[1] + s0[2] * s0[2]);
        const double l1 = sqrt(s1[0] * s1[0] + s1[1] * s1[1] + s1[2] * s1[2]);
        const double l2 = sqrt(s2[0] * s2[0] + s2[1] * s2[1] + s2[2] * s2[2]);
        double ang;
        if (slot == 0) ang = acos(-(s2[0] * s0[0] + s2[1] * s0[1] + s2[2] * s0[2]) / (l2 * l0));
        else if (slot == 1) ang = acos(-(s0[0] * s1[0] + s0[1] * s1[1] + s0[2] * s1[2]) / (l0 * l1));
        else ang = acos(-(s1[0] * s2[0] + s1[1] * s2[1] + s1[2] * s2[2]) / (l1 * l2));
        acc += -ang;
    }
    out[n] = acc;
}

__global__ void k_kinetic(const DevMesh m, const DevState s, int parity, double* ke) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const size_t N = m.N;
    const double* v = vel_buf(s, parity);
    const double vx = v[n], vy = v[N + n], vz = v[2 * N + n];
    ke[n] = 0.5 * m.mass[n] * (vx * vx + vy * vy + vz * vz);
}

// Neumaier-compensated sums: pass 1, one fixed slice per block; pass 2, one
// thread folds the block partials in order.
constexpr int kSumBlocks = 256;

__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__global__ void k_comp_sum_pass1(const double* x, int n, double* partial) {
    __shared__ double ss[256], sc[256];
    const int per_block = (n + gridDim.x - 1) / gridDim.x;
    const int lo = blockIdx.x * per_block, hi = min(n, lo + per_block);
    double s = 0.0, c = 0.0;
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) neumaier_add(s, c, x[i]);
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, C = 0.0;
        for (int k = 0; k < (int)blockDim.x; ++k) {
            neumaier_add(S, C, ss[k]);
            C += sc[k];
        }
        partial[2 * blockIdx.x] = S;
        partial[2 * blockIdx.x + 1] = C;
    }
}

__global__ void k_comp_sum_pass2(const double* partial, int nb, double* out) {
    double S = 0.0, C = 0.0;
    for (int b = 0; b < nb; ++b) {
        neumaier_add(S, C, partial[2 * b]);
        C += partial[2 * b + 1];
    }
    *out = S + C;
}

__global__ void k_chunk_end(DevError* e, int len) { e->base += len; }

inline int blocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

cudaError_t launch_node_update(const DevMesh& m, const DevState& s, const StepScalars& sc, int mixed,
                               cudaStream_t st) {
    const int nb = blocks_for(m.N, kNodeBlock);
    (void)mixed;
    if (mixed) k_node_update<true><<<nb, kNodeBlock, 0, st>>>(m, s, sc);
    else k_node_update<false><<<nb, kNodeBlock, 0, st>>>(m, s, sc);
    return cudaGetLastError();
}

cudaError_t launch_surface_derivs(const DevMesh& m, const DevState& s, int parity, cudaStream_t st) {
    k_surface_derivs<<<blocks_for(m.T, 128), 128, 0, st>>>(m, s, parity);
    return cudaGetLastError();
}
cudaError_t launch_forces_from_cq(const DevMesh& m, const DevState& s, int write_dE, cudaStream_t st) {
    k_forces_from_cq<<<blocks_for(m.T, 128), 128, 0, st>>>(m, s, write_dE);
    return cudaGetLastError();
}
cudaError_t launch_gather_forces(const DevMesh& m, const DevState& s, cudaStream_t st) {
    k_gather_forces<<<blocks_for(m.N, 256), 256, 0, st>>>(m, s);
    return cudaGetLastError();
}
cudaError_t launch_damping(const DevMesh& m, const DevState& s, int parity, double damping, double rho_hh,
                           cudaStream_t st) {
    k_damping<<<blocks_for(m.N, 256), 256, 0, st>>>(m, s, parity, damping, rho_hh);
    return cudaGetLastError();
}
cudaError_t launch_constraints(const DevMesh& m, const DevState& s, cudaStream_t st) {
    k_constraints<<<blocks_for(m.N, 256), 256, 0, st>>>(m, s);
    return cudaGetLastError();
}
cudaError_t launch_equilibrium(const DevMesh& m, const DevState& s, int parity, cudaStream_t st) {
    k_equilibrium<<<blocks_for(m.N, kNodeBlock), kNodeBlock, 0, st>>>(m, s, parity);
    return cudaGetLastError();
}
cudaError_t launch_guard(const DevMesh& m, const DevState& s, double lim, cudaStream_t st) {
    k_guard<<<blocks_for(3LL * m.N, 256), 256, 0, st>>>(m, s, lim);
    return cudaGetLastError();
}
cudaError_t launch_advance(const DevMesh& m, const DevState& s, int parity, double dt, double damping, double rho_hh,
                           int gd, cudaStream_t st) {
    k_advance<<<blocks_for(3LL * m.N, 256), 256, 0, st>>>(m, s, parity, dt, damping, rho_hh, gd);
    return cudaGetLastError();
}
cudaError_t launch_dialling(const DevMesh& m, int protocol, double dial, double spacing, int from_ansatz,
                            cudaStream_t st) {
    k_dialling<<<blocks_for(m.T, 128), 128, 0, st>>>(m, protocol, dial, spacing, from_ansatz);
    return cudaGetLastError();
}
cudaError_t launch_a_b_normals(const DevMesh& m, const DevState& s, double* a, double* b, double* n,
                               cudaStream_t st) {
    k_a_b_normals<<<blocks_for(m.T, 128), 128, 0, st>>>(m, s, a, b, n);
    return cudaGetLastError();
}
cudaError_t launch_output_tri(const DevMesh& m, const DevState& s, double* curv, double* edens, double* strain,
                              double* stress, double* tri_energy, cudaStream_t st) {
    k_output_tri<<<blocks_for(m.T, 128), 128, 0, st>>>(m, s, curv, edens, strain, stress, tri_energy);
    return cudaGetLastError();
}
cudaError_t launch_angle_deficits(const DevMesh& m, const DevState& s, int parity, double* out, cudaStream_t st) {
    k_angle_deficits<<<blocks_for(m.N, 256), 256, 0, st>>>(m, s, parity, out);
    return cudaGetLastError();
}
cudaError_t launch_kinetic(const DevMesh& m, const DevState& s, int parity, double* ke, cudaStream_t st) {
    k_kinetic<<<blocks_for(m.N, 256), 256, 0, st>>>(m, s, parity, ke);
    return cudaGetLastError();
}
cudaError_t launch_chunk_end(const DevState& s, int len, cudaStream_t st) {
    k_chunk_end<<<1, 1, 0, st>>>(s.err, len);
    return cudaGetLastError();
}
cudaError_t launch_comp_sum(const double* x, int n, double* partial, double* out, cudaStream_t st) {
    const int nb = n < kSumBlocks * 256 ? max(1, blocks_for(n, 256)) : kSumBlocks;
    k_comp_sum_pass1<<<nb, 256, 0, st>>>(x, n, partial);
    k_comp_sum_pass2<<<1, 1, 0, st>>>(partial, nb, out);
    return cudaGetLastError();
}

void build_sell(int N, const int* off, const int* ent, std::vector<int>& sell_off, std::vector<int>& sell_ent) {
    const int W = (N + 31) / 32;
    sell_off.assign(W + 1, 0);
    for (int w = 0; w < W; ++w) {
        int width = 0;
        for (int l = 0; l < 32 && 32 * w + l < N; ++l) width = std::max(width, off[32 * w + l + 1] - off[32 * w + l]);
        sell_off[w + 1] = sell_off[w] + 32 * width;
    }
    sell_ent.assign((size_t)sell_off[W], -1);
    for (int w = 0; w < W; ++w)
        for (int l = 0; l < 32 && 32 * w + l < N; ++l) {
            const int n = 32 * w + l;
            for (int k = off[n]; k < off[n + 1]; ++k) sell_ent[(size_t)sell_off[w] + 32 * (k - off[n]) + l] = ent[k];
        }
}

}  // namespace msb
