// Drives the reference's own per-step functions (compiled unmodified from
// source_files/ against eigen_shim/) through the ref_* C ABI of oracle.h.
// TEST INFRASTRUCTURE ONLY.
//
// The per-step sequence follows source_files/main.cpp:308-474; the mesh
// set-up is shared with the product (same patch nodes and patch matrices),
// but the sparse derivative matrix and the dof masses are built by the
// reference's calc_deriv_mats and calc_dof_masses.
#include <omp.h>

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "Node_Class.hpp"
#include "Out_Stream_Class.hpp"
#include "Stuff_Class.hpp"
#include "Tri_Class.hpp"
#include "advance_dynamics.hpp"
#include "Edge_Class.hpp"
#include "calc_a_comps_and_b_comps_and_normals.hpp"
#include "calc_char_mechanics_scales.hpp"
#include "calc_damping_factor.hpp"
#include "calc_dialling_procedure_params.hpp"
#include "calc_long_timescales.hpp"
#include "calc_mesh_info.hpp"
#include "calc_steps_between_outputs.hpp"
#include "calc_timestep.hpp"
#include "perturb_node_positions_with_noise.hpp"
#include "read_settings.hpp"
#include "read_vtk_data.hpp"
#include "set_up_patch_fitting.hpp"
#include "calc_angle_deficits.hpp"
#include "calc_curvatures.hpp"
#include "calc_deformation_forces.hpp"
#include "calc_deriv_mats.hpp"
#include "calc_dof_masses.hpp"
#include "calc_energies.hpp"
#include "calc_energy_densities.hpp"
#include "calc_non_deformation_forces.hpp"
#include "calc_strains.hpp"
#include "calc_stresses.hpp"
#include "calc_surface_derivs.hpp"
#include "do_dialling.hpp"
#include "impose_constraints.hpp"
#include "is_at_equilibrium.hpp"
#include "oracle.h"

// do_dialling.cpp compiled once more per protocol 2..5 with that protocol's
// block enabled (the reference selects protocols by editing that file).
#define MS_DECLARE_DIALLING(NAME)                                                                               \
    void NAME(Eigen::Matrix<double, Eigen::Dynamic, 3>& abar_comps,                                             \
              Eigen::Matrix<double, Eigen::Dynamic, 3>& bbar_comps,                                             \
              Eigen::Matrix<double, Eigen::Dynamic, 1>& def_thicknesses,                                        \
              Eigen::Matrix<double, Eigen::Dynamic, 1>& def_shear_moduli, double dial_factor,                   \
              const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic>& abar_info,                           \
              const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic>& bbar_info,                           \
              const Eigen::Matrix<double, Eigen::Dynamic, 3>& a_comps_at_zero_dial_factor,                      \
              const Eigen::Matrix<double, Eigen::Dynamic, 3>& b_comps_at_zero_dial_factor,                      \
              const std::vector<Tri_Class>& triangles, const std::vector<Node_Class>& nodes,                    \
              const Eigen::Matrix<double, Eigen::Dynamic, 1>& dofs,                                             \
              const Eigen::Matrix<double, Eigen::Dynamic, 3>& normals, Out_Stream_Class& log,                   \
              const Stuff_Class& stuff);
MS_DECLARE_DIALLING(do_dialling_protocol2)
MS_DECLARE_DIALLING(do_dialling_protocol3)
MS_DECLARE_DIALLING(do_dialling_protocol4)
MS_DECLARE_DIALLING(do_dialling_protocol5)

namespace {

using VecX = Eigen::Matrix<double, Eigen::Dynamic, 1>;
using MatX3 = Eigen::Matrix<double, Eigen::Dynamic, 3>;
using MatX2 = Eigen::Matrix<double, Eigen::Dynamic, 2>;
using MatXX = Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic>;
using Sparse = Eigen::SparseMatrix<double, Eigen::RowMajor>;

struct Ctx {
    Stuff_Class stuff;
    std::vector<Node_Class> nodes;
    std::vector<Tri_Class> tris;
    Sparse D, DT;
    VecX dofs, vel, forces, cq, dE, masses, thick, shear;
    MatX3 abar, bbar, a0, b0, normals;
    MatXX abar_info, bbar_info;
    Out_Stream_Class log;
    int protocol = 1;
};

void copy_rowmajor(MatXX& m, const double* src, int rows, int cols) {
    m.resize(rows, cols);
    for (int i = 0; i < rows; ++i)
        for (int j = 0; j < cols; ++j) m(i, j) = src[(size_t)i * cols + j];
}

void dial(Ctx& c, double f) {
    auto* fn = c.protocol == 2   ? &do_dialling_protocol2
               : c.protocol == 3 ? &do_dialling_protocol3
               : c.protocol == 4 ? &do_dialling_protocol4
               : c.protocol == 5 ? &do_dialling_protocol5
                                 : &do_dialling;
    fn(c.abar, c.bbar, c.thick, c.shear, f, c.abar_info, c.bbar_info, c.a0, c.b0, c.tris, c.nodes, c.dofs,
       c.normals, c.log, c.stuff);
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n); }

// The reference's own set-up sequence (main.cpp:91-209): settings, mesh file,
// topology, patch fitting, derivative matrix, masses, scales, timestep and
// dialling schedule, initial noise.  Outputs (any may be NULL): patch T x 6,
// mat2 T x 18, node masses N, initial dofs 3N (after noise), and
// scal[14] = {sample_char_length, approx_min_tri_size, min_ref_thickness,
// char_force_scale, char_speed_scale, char_long_time, damping_factor(pref 1),
// timestep, timesteps_per_dial_phase, timesteps_between_equil_checks,
// total_ref_area, num_edges, num_boundary_nodes, damping_factor(pref 2)}.
// Returns 0, or 1 with the exception text in err (len bytes).
int ref_setup_from_files(const char* settings, const char* vtk, int* N_out, int* T_out, int32_t* patch,
                         double* mat2, double* masses, double* dofs0, double* scal, char* err, int len) {
    return ref_setup_full(settings, vtk, N_out, T_out, patch, mat2, masses, dofs0, scal, nullptr, nullptr, nullptr,
                          nullptr, nullptr, nullptr, err, len);
}

// As ref_setup_from_files, plus what ref_create needs besides: the flat
// reference positions as read from the mesh file (N x 3 row-major), per
// triangle ref_area, ref_thickness and ref_shear_modulus (T each, from
// calc_mesh_info and read_vtk_data), and per node is_constrained and
// is_boundary (N each).  Any output may be NULL.
int ref_setup_full(const char* settings, const char* vtk, int* N_out, int* T_out, int32_t* patch, double* mat2,
                   double* masses, double* dofs0, double* scal, double* ref_pos, double* area, double* thick,
                   double* shear, uint8_t* fixed, uint8_t* boundary, char* err, int len) {
    try {
        Stuff_Class st;
        Out_Stream_Class log;
        log.set_output_filepath("/dev/null");
        st.settings_filepath = settings;
        st.ref_data_filepath = vtk;
        st.ansatz_file_was_given = false;
        read_settings(st, log);
        std::vector<Node_Class> nodes;
        Eigen::Matrix<double, Eigen::Dynamic, 3> P;
        std::vector<Eigen::Vector3d> ans;
        std::vector<Tri_Class> tris;
        MatXX ai, bi;
        double d0 = 0.0;
        read_vtk_data(nodes, P, ans, tris, ai, bi, st, d0, log);
        std::vector<Edge_Class> edges;
        calc_mesh_info(nodes, P, tris, edges, st, log);
        set_up_patch_fitting(nodes, P, tris, st, log);
        Sparse D(st.num_continuum_quantities, st.num_dofs), DT(st.num_dofs, st.num_continuum_quantities);
        calc_deriv_mats(D, DT, P, tris, st, log);
        VecX m(st.num_dofs, 1);
        calc_dof_masses(m, tris, st, log);
        calc_char_mechanics_scales(tris, st);
        calc_long_timescales(st, log);
        calc_damping_factor(st.damping_prefactor_2, st, log);
        const double damp2 = st.damping_factor;
        calc_damping_factor(st.damping_prefactor_1, st, log);
        calc_timestep(st, log);
        calc_steps_between_outputs(st, log);
        calc_dialling_procedure_params(st, log);
        if (ref_pos)
            for (int n = 0; n < st.num_nodes; ++n)
                for (int k = 0; k < 3; ++k) ref_pos[3 * (size_t)n + k] = P(n, k);
        perturb_node_positions_with_noise(P, st);
        for (int t = 0; t < st.num_tris; ++t) {
            if (area) area[t] = tris[t].ref_area;
            if (thick) thick[t] = tris[t].ref_thickness;
            if (shear) shear[t] = tris[t].ref_shear_modulus;
        }
        for (int n = 0; n < st.num_nodes; ++n) {
            if (fixed) fixed[n] = nodes[n].is_constrained ? 1 : 0;
            if (boundary) boundary[n] = nodes[n].is_boundary ? 1 : 0;
        }
        if (N_out) *N_out = st.num_nodes;
        if (T_out) *T_out = st.num_tris;
        for (int t = 0; t < st.num_tris; ++t) {
            for (int v = 0; v < 3; ++v) {
                if (patch) patch[6 * (size_t)t + v] = tris[t].vertex_ids[v];
                if (patch) patch[6 * (size_t)t + 3 + v] = tris[t].non_vertex_patch_nodes_ids[v];
            }
            for (int r = 0; r < 6; ++r)
                for (int k = 0; k < 3; ++k)
                    if (mat2) mat2[18 * (size_t)t + 3 * r + k] = tris[t].mat_for_patch_2nd_derivs(r, k);
        }
        for (int n = 0; n < st.num_nodes; ++n) {
            if (masses) masses[n] = m(n);
            for (int k = 0; k < 3; ++k)
                if (dofs0) dofs0[(size_t)k * st.num_nodes + n] = P(n, k);
        }
        if (scal) {
            const double v[14] = {st.sample_char_length, st.approx_min_tri_size, st.min_ref_thickness,
                                  st.char_force_scale, st.char_speed_scale, st.char_long_time, st.damping_factor,
                                  st.timestep, (double)st.timesteps_per_dial_phase,
                                  (double)st.timesteps_between_equil_checks, st.total_ref_area, (double)st.num_edges,
                                  (double)st.num_boundary_nodes, damp2};
            for (int k = 0; k < 14; ++k) scal[k] = v[k];
        }
        return 0;
    } catch (const std::exception& e) {
        if (err && len > 0) {
            std::strncpy(err, e.what(), len - 1);
            err[len - 1] = 0;
        }
        return 1;
    }
}

void* ref_create(int N, int T, const double* ref_pos, const int32_t* patch, const double* mat2, const double*,
                 const double*, const double* area, const double* thick, const double* shear, const uint8_t* fixed,
                 const uint8_t* boundary, const double* scal) {
    Ctx* c = new Ctx();
    c->log.set_output_filepath("/dev/null");
    Stuff_Class& s = c->stuff;
    s.num_nodes = N;
    s.num_tris = T;
    s.num_dofs = 3 * N;
    s.num_continuum_quantities = 15 * T;
    s.def_poisson_ratio = scal[0];
    s.bend_stiffening_scale_factor = scal[1];
    s.ref_density = scal[2];
    s.min_ref_thickness = scal[3];
    s.char_force_scale = scal[4];
    s.char_speed_scale = scal[5];
    s.force_to_char_force_ratio_equil_threshold = scal[6];
    s.speed_to_char_speed_ratio_equil_threshold = scal[7];
    s.slide_stiffness_prefactor = 0.0;
    s.slide_friction_coefficent = 0.0;
    s.slide_speed_prefactor = 0.0;
    s.upper_slide_z_coord = 1e300;
    s.lower_slide_z_coord = -1e300;
    s.upper_slide_tot_vert_force = 0.0;
    s.lower_slide_tot_vert_force = 0.0;
    s.sample_char_length = 1.0;
    s.bend_long_time = 1.0;
    s.using_gradient_descent_dynamics = false;
    s.dialling_from_ansatz_rather_than_ref_state = false;
    s.dial_factors_to_hold_at_spacing = 1.0;
    c->nodes.resize(N);
    for (int n = 0; n < N; ++n) {
        c->nodes[n].id = n;
        c->nodes[n].is_constrained = fixed[n] != 0;
        c->nodes[n].is_boundary = boundary ? boundary[n] != 0 : false;
    }
    Eigen::Matrix<double, Eigen::Dynamic, 3> P(N, 3);
    for (int n = 0; n < N; ++n)
        for (int k = 0; k < 3; ++k) P(n, k) = ref_pos[3 * (size_t)n + k];
    c->tris.resize(T);
    for (int t = 0; t < T; ++t) {
        Tri_Class& tr = c->tris[t];
        tr.id = t;
        for (int v = 0; v < 3; ++v) {
            tr.vertex_ids[v] = patch[6 * (size_t)t + v];
            tr.non_vertex_patch_nodes_ids[v] = patch[6 * (size_t)t + 3 + v];
        }
        for (int k = 0; k < 3; ++k)
            tr.ref_centroid(k) = (P(tr.vertex_ids[0], k) + P(tr.vertex_ids[1], k) + P(tr.vertex_ids[2], k)) / 3.0;
        for (int r = 0; r < 6; ++r)
            for (int k = 0; k < 3; ++k) tr.mat_for_patch_2nd_derivs(r, k) = mat2[18 * (size_t)t + 3 * r + k];
        tr.ref_area = area[t];
        tr.ref_thickness = thick[t];
        tr.ref_shear_modulus = shear[t];
    }
    c->D = Sparse(15 * T, 3 * N);
    c->DT = Sparse(3 * N, 15 * T);
    calc_deriv_mats(c->D, c->DT, P, c->tris, s, c->log);
    c->masses.resize(3 * N, 1);
    calc_dof_masses(c->masses, c->tris, s, c->log);
    c->dofs.resize(3 * N, 1);
    c->vel.resize(3 * N, 1);
    c->forces.resize(3 * N, 1);
    c->cq.resize(15 * T, 1);
    c->dE.resize(15 * T, 1);
    c->thick.resize(T, 1);
    c->shear.resize(T, 1);
    for (int t = 0; t < T; ++t) {
        c->thick(t) = thick[t];
        c->shear(t) = shear[t];
    }
    for (MatX3* m : {&c->abar, &c->bbar, &c->a0, &c->b0, &c->normals}) m->resize(T, 3);
    c->a0.fill(1);
    c->a0.col(1).fill(0);
    c->b0.fill(0);
    c->abar = c->a0;
    c->bbar = c->b0;
    c->dofs.fill(0);
    c->vel.fill(0);
    c->forces.fill(0);
    return c;
}

void ref_destroy(void* p) { delete static_cast<Ctx*>(p); }

int ref_set_programmed(void* p, int protocol, const double* ai, int ka, const double* bi, int kb, double spacing,
                       int from_ansatz) {
    Ctx& c = *static_cast<Ctx*>(p);
    if (protocol < 1 || protocol > 5) return 8;
    // Protocols 1 and 2 combine whole T x 3 matrices; 3..5 read columns.
    const int need_a[6] = {0, 3, 3, 3, 13, 1};
    if ((protocol <= 2 && (ka != 3 || kb != 3)) || ka < need_a[protocol]) return 1;
    c.protocol = protocol;
    copy_rowmajor(c.abar_info, ai, c.stuff.num_tris, ka);
    copy_rowmajor(c.bbar_info, bi, c.stuff.num_tris, kb);
    c.stuff.dial_factors_to_hold_at_spacing = spacing;
    c.stuff.dialling_from_ansatz_rather_than_ref_state = from_ansatz != 0;
    return 0;
}

void ref_set_zero_dial_state(void* p, const double* a0, const double* b0) {
    Ctx& c = *static_cast<Ctx*>(p);
    const int T = c.stuff.num_tris;
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k) {
            c.a0(t, k) = a0 ? a0[3 * (size_t)t + k] : (k == 1 ? 0.0 : 1.0);
            c.b0(t, k) = b0 ? b0[3 * (size_t)t + k] : 0.0;
        }
}

void ref_set_state(void* p, const double* dofs, const double* vel) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int d = 0; d < c.stuff.num_dofs; ++d) {
        c.dofs(d) = dofs[d];
        c.vel(d) = vel ? vel[d] : 0.0;
    }
}

void ref_get_state(void* p, double* dofs, double* vel) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int d = 0; d < c.stuff.num_dofs; ++d) {
        if (dofs) dofs[d] = c.dofs(d);
        if (vel) vel[d] = c.vel(d);
    }
}

void ref_get_forces(void* p, double* f) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int d = 0; d < c.stuff.num_dofs; ++d) f[d] = c.forces(d);
}

void ref_do_dialling(void* p, double f) { dial(*static_cast<Ctx*>(p), f); }

void ref_get_programmed(void* p, double* abar, double* bbar) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int t = 0; t < c.stuff.num_tris; ++t)
        for (int k = 0; k < 3; ++k) {
            if (abar) abar[3 * (size_t)t + k] = c.abar(t, k);
            if (bbar) bbar[3 * (size_t)t + k] = c.bbar(t, k);
        }
}

void ref_surface_derivs(void* p, double* cq) {
    Ctx& c = *static_cast<Ctx*>(p);
    calc_surface_derivs(c.cq, c.D, c.dofs);
    if (cq) std::memcpy(cq, c.cq.data(), sizeof(double) * 15 * (size_t)c.stuff.num_tris);
}

void ref_a_b_normals(void* p, double* a, double* b, double* n) {
    Ctx& c = *static_cast<Ctx*>(p);
    MatX3 A(c.stuff.num_tris, 3), B(c.stuff.num_tris, 3);
    calc_a_comps_and_b_comps_and_normals(A, B, c.normals, c.cq, c.stuff);
    for (int t = 0; t < c.stuff.num_tris; ++t)
        for (int k = 0; k < 3; ++k) {
            a[3 * (size_t)t + k] = A(t, k);
            b[3 * (size_t)t + k] = B(t, k);
            n[3 * (size_t)t + k] = c.normals(t, k);
        }
}

void ref_deformation_forces(void* p, double* f, double* dE) {
    Ctx& c = *static_cast<Ctx*>(p);
    calc_deformation_forces(c.forces, c.dE, c.cq, c.shear, c.thick, c.abar, c.bbar, c.DT, c.tris, c.stuff, c.log);
    if (f) ref_get_forces(p, f);
    if (dE) std::memcpy(dE, c.dE.data(), sizeof(double) * 15 * (size_t)c.stuff.num_tris);
}

void ref_non_deformation_forces(void* p, double damping, int gd) {
    Ctx& c = *static_cast<Ctx*>(p);
    c.stuff.damping_factor = damping;
    c.stuff.using_gradient_descent_dynamics = gd != 0;
    calc_non_deformation_forces(c.forces, c.vel, c.dofs, c.masses, c.stuff);
}

void ref_impose_constraints(void* p) {
    Ctx& c = *static_cast<Ctx*>(p);
    impose_constraints(c.nodes, c.dofs, c.vel, c.forces, c.tris, c.stuff);
}

int ref_is_at_equilibrium(void* p, double* out4) {
    Ctx& c = *static_cast<Ctx*>(p);
    const bool eq = is_at_equilibrium(c.forces, c.vel, c.stuff, c.log);
    if (out4) {
        // is_at_equilibrium only logs its maxima; recompute them the same way.
        const int N = c.stuff.num_nodes;
        double mf = -1, mv = -1;
        int nf = 0, nv = 0;
        for (int n = 0; n < N; ++n) {
            Eigen::Vector3d f = {c.forces(n), c.forces(n + N), c.forces(n + 2 * N)};
            Eigen::Vector3d v = {c.vel(n), c.vel(n + N), c.vel(n + 2 * N)};
            if (f.norm() > mf) { mf = f.norm(); nf = n; }
            if (v.norm() > mv) { mv = v.norm(); nv = n; }
        }
        out4[0] = mf;
        out4[1] = mv;
        out4[2] = nf;
        out4[3] = nv;
    }
    return eq ? 1 : 0;
}

int ref_advance_dynamics(void* p, double dt, double damping, int gd, int64_t* bad_dof, double* bad_force) {
    Ctx& c = *static_cast<Ctx*>(p);
    c.stuff.timestep = dt;
    c.stuff.damping_factor = damping;
    c.stuff.using_gradient_descent_dynamics = gd != 0;
    try {
        advance_dynamics(c.dofs, c.vel, c.forces, c.masses, c.stuff, c.log);
    } catch (const std::runtime_error&) {
        for (int d = 0; d < c.stuff.num_dofs; ++d)
            if (!(std::fabs(c.forces(d)) < 50000.0 * c.stuff.char_force_scale)) {
                if (bad_dof) *bad_dof = d;
                if (bad_force) *bad_force = c.forces(d);
                break;
            }
        return 3;
    }
    return 0;
}

int ref_step_n(void* p, int n, const double* dials, double dt, double damping, int gd, int* done) {
    Ctx& c = *static_cast<Ctx*>(p);
    for (int i = 0; i < n; ++i) {
        if (done) *done = i;
        calc_surface_derivs(c.cq, c.D, c.dofs);
        if (dials) dial(c, dials[i]);
        calc_deformation_forces(c.forces, c.dE, c.cq, c.shear, c.thick, c.abar, c.bbar, c.DT, c.tris, c.stuff, c.log);
        ref_non_deformation_forces(p, damping, gd);
        impose_constraints(c.nodes, c.dofs, c.vel, c.forces, c.tris, c.stuff);
        if (ref_advance_dynamics(p, dt, damping, gd, nullptr, nullptr) != 0) return 3;
    }
    if (done) *done = n;
    return 0;
}

void ref_output_quantities(void* p, double* curv, double* edens, double* strains, double* stresses, double* deficits,
                           double* energies) {
    Ctx& c = *static_cast<Ctx*>(p);
    const int T = c.stuff.num_tris, N = c.stuff.num_nodes;
    calc_surface_derivs(c.cq, c.D, c.dofs);
    MatX3 A(T, 3), B(T, 3);
    calc_a_comps_and_b_comps_and_normals(A, B, c.normals, c.cq, c.stuff);
    MatX2 cu(T, 2), ed(T, 2);
    VecX ad(N, 1), st(T, 1);
    Eigen::Matrix<double, Eigen::Dynamic, 8> ss(T, 8);
    std::vector<double> en(3);
    calc_curvatures(cu, c.cq, B, c.stuff);
    calc_angle_deficits(ad, c.dofs, c.nodes, c.tris, c.stuff);
    calc_energy_densities(ed, A, B, c.abar, c.bbar, c.shear, c.thick, c.stuff, c.log);
    calc_energies(en, ed, c.vel, c.masses, c.tris, c.stuff);
    calc_stresses(ss, c.cq, c.abar, c.bbar, c.shear, c.thick, c.tris, c.stuff, c.log);
    calc_strains(st, c.cq, A, c.abar, c.stuff);
    for (int t = 0; t < T; ++t) {
        for (int k = 0; k < 2; ++k) {
            if (curv) curv[2 * (size_t)t + k] = cu(t, k);
            if (edens) edens[2 * (size_t)t + k] = ed(t, k);
        }
        if (strains) strains[t] = st(t);
        for (int k = 0; k < 8; ++k)
            if (stresses) stresses[8 * (size_t)t + k] = ss(t, k);
    }
    for (int n = 0; n < N; ++n)
        if (deficits) deficits[n] = ad(n);
    if (energies)
        for (int k = 0; k < 3; ++k) energies[k] = en[k];
}

}  // extern "C"
