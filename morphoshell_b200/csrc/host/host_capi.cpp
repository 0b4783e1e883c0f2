// Host C ABI (include/morphoshell_host.h): the one-off set-up of main.cpp:74-238
// and the dynamics loop of main.cpp:269-508, driving the GPU through the
// per-step C ABI of include/morphoshell_gpu.h.
#include <chrono>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <iomanip>
#include <memory>

#include "../../../include/morphoshell_host.h"
#include "host.hpp"

using namespace msb;

struct msh_model {
    Stuff stuff;
    std::vector<Node> nodes;
    std::vector<Tri> tris;
    std::vector<Edge> edges;
    DMat ref_positions;   // flat reference state
    DMat init_positions;  // after noise / ansatz
    DMat abar_info, bbar_info;
    std::vector<std::array<double, 3>> ansatz;
    double dial_factor_to_start_from = 0.0;
    double damping_factor_1 = 0, damping_factor_2 = 0;
    // flattened tables for ms_create
    std::vector<int32_t> patch_ids;
    std::vector<double> coeffs, area, thick, shear, mass;
    std::vector<uint8_t> fixed, boundary;
};

namespace {

thread_local std::string g_err;

int set_err(const std::string& s) {
    g_err = s;
    return 1;
}

void soa_from(const DMat& P, double* dofs) {
    const int N = P.rows;
    for (int n = 0; n < N; ++n)
        for (int c = 0; c < 3; ++c) dofs[(size_t)c * N + n] = P(n, c);
}

}  // namespace

extern "C" {

const char* msh_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace {

// Mesh data handed over in memory instead of read from the input VTK file.
struct ArrayMesh {
    int N, T;
    const double* pos;
    const int32_t* tris;
    const double* abar_info;
    int ka;
    const double* bbar_info;
    int kb;
    const double* thick;
    const double* shear;
    const uint8_t* constrained;
};

// Fills what read_vtk_data would (read_vtk_data.cpp:84-371), including the
// uniform thickness / modulus overrides of the settings file.
void fill_from_arrays(msh_model& m, const ArrayMesh& a) {
    Stuff& st = m.stuff;
    if (a.N <= 0 || a.T <= 0 || a.ka <= 0 || a.kb <= 0)
        throw std::runtime_error("Error: mesh arrays have a non-positive size.");
    st.num_nodes = a.N;
    st.num_tris = a.T;
    m.nodes.assign(a.N, Node());
    m.ref_positions.resize(a.N, 3);
    for (int n = 0; n < a.N; ++n) {
        m.nodes[n].id = n;
        m.nodes[n].is_constrained = a.constrained ? a.constrained[n] != 0 : false;
        for (int c = 0; c < 3; ++c) m.ref_positions(n, c) = a.pos[3 * (size_t)n + c];
    }
    m.tris.assign(a.T, Tri());
    bool found_zero = false;
    for (int t = 0; t < a.T; ++t) {
        m.tris[t].id = t;
        for (int v = 0; v < 3; ++v) {
            const int id = a.tris[3 * (size_t)t + v];
            if (id < 0 || id >= a.N) throw std::runtime_error("Error: a triangle vertex id is out of range.");
            found_zero |= id == 0;
            m.tris[t].vertex_ids[v] = id;
        }
        m.tris[t].ref_thickness = st.ref_thickness_if_uniform > 0 ? st.ref_thickness_if_uniform : a.thick[t];
        m.tris[t].ref_shear_modulus =
            st.ref_shear_modulus_if_uniform > 0 ? st.ref_shear_modulus_if_uniform : a.shear[t];
    }
    if (!found_zero) throw std::runtime_error("Error: MorphoShell requires node ids starting from 0.");
    m.abar_info.resize(a.T, a.ka);
    std::memcpy(m.abar_info.v.data(), a.abar_info, sizeof(double) * (size_t)a.T * a.ka);
    m.bbar_info.resize(a.T, a.kb);
    std::memcpy(m.bbar_info.v.data(), a.bbar_info, sizeof(double) * (size_t)a.T * a.kb);
}

int load_common(const char* settings_path, const char* vtk_path, const ArrayMesh* arrays, const char* ansatz_path,
                int flags, msh_model** out) {
    if (!settings_path || (!vtk_path && !arrays) || !out) return set_err("null argument");
    *out = nullptr;
    auto m = std::make_unique<msh_model>();
    Stuff& st = m->stuff;
    Log log;
    log.set_quiet(flags & 1);
    try {
        st.settings_filepath = settings_path;
        st.ref_data_filepath = vtk_path ? vtk_path : "in-memory mesh";
        st.ansatz_file_was_given = ansatz_path != nullptr;
        st.ansatz_filepath = ansatz_path ? ansatz_path : "no_ansatz_file";
        read_settings(st, log);
        if (arrays) {
            if (st.ansatz_file_was_given) throw std::runtime_error("Error: in-memory meshes take no ansatz file.");
            fill_from_arrays(*m, *arrays);
        } else {
            read_vtk_data(m->nodes, m->ref_positions, m->ansatz, m->tris, m->abar_info, m->bbar_info, st,
                          m->dial_factor_to_start_from, log);
        }
        if (st.dialling_from_ansatz_rather_than_ref_state) m->dial_factor_to_start_from = 0.0;
        calc_mesh_info(m->nodes, m->ref_positions, m->tris, m->edges, st, log);
        if (flags & 4) {
            set_up_patches_on_device(m->nodes, m->ref_positions, m->tris, st, m->coeffs, log);
        } else {
            set_up_patch_fitting(m->nodes, m->ref_positions, m->tris, st, log);
            calc_deriv_coeffs(m->coeffs, m->ref_positions, m->tris, st);
        }
        calc_dof_masses(m->mass, m->tris, st);
        calc_char_mechanics_scales(m->tris, st);
        calc_long_timescales(st, log);
        calc_damping_factor(st.damping_prefactor_2, st, log);
        m->damping_factor_2 = st.damping_factor;
        calc_damping_factor(st.damping_prefactor_1, st, log);
        m->damping_factor_1 = st.damping_factor;
        calc_timestep(st, log);
        calc_steps_between_outputs(st, log);
        calc_dialling_procedure_params(st, log);
        m->init_positions = m->ref_positions;
        if (!(flags & 2)) perturb_node_positions_with_noise(m->init_positions, st);
        if (st.ansatz_file_was_given)
            for (int n = 0; n < st.num_nodes; ++n)
                for (int c = 0; c < 3; ++c) m->init_positions(n, c) = m->ansatz.at(n)[c];
        initialize_glass_slides(m->init_positions, st);
    } catch (const std::exception& e) {
        return set_err(e.what());
    }
    const int T = st.num_tris, N = st.num_nodes;
    m->patch_ids.resize(6ULL * T);
    m->area.resize(T);
    m->thick.resize(T);
    m->shear.resize(T);
    for (int t = 0; t < T; ++t) {
        for (int v = 0; v < 3; ++v) {
            m->patch_ids[6ULL * t + v] = m->tris[t].vertex_ids[v];
            m->patch_ids[6ULL * t + 3 + v] = m->tris[t].non_vertex_patch_nodes_ids[v];
        }
        m->area[t] = m->tris[t].ref_area;
        m->thick[t] = m->tris[t].ref_thickness;
        m->shear[t] = m->tris[t].ref_shear_modulus;
    }
    m->fixed.resize(N);
    m->boundary.resize(N);
    for (int n = 0; n < N; ++n) {
        m->fixed[n] = m->nodes[n].is_constrained ? 1 : 0;
        m->boundary[n] = m->nodes[n].is_boundary ? 1 : 0;
    }
    *out = m.release();
    return 0;
}

}  // namespace

extern "C" {

int msh_load(const char* settings_path, const char* vtk_path, const char* ansatz_path, int flags, msh_model** out) {
    return load_common(settings_path, vtk_path, nullptr, ansatz_path, flags, out);
}

int msh_build(const char* settings_path, int32_t num_nodes, int32_t num_tris, const double* positions,
              const int32_t* tri_vertex_ids, const double* abar_info, int32_t ka, const double* bbar_info, int32_t kb,
              const double* ref_thicknesses, const double* ref_shear_moduli, const uint8_t* constrained, int flags,
              msh_model** out) {
    if (!positions || !tri_vertex_ids || !abar_info || !bbar_info) return set_err("null argument");
    std::vector<double> ones(num_tris > 0 ? num_tris : 0, 1.0);
    ArrayMesh a{num_nodes, num_tris, positions, tri_vertex_ids, abar_info, ka, bbar_info, kb,
                ref_thicknesses ? ref_thicknesses : ones.data(), ref_shear_moduli ? ref_shear_moduli : ones.data(),
                constrained};
    return load_common(settings_path, nullptr, &a, nullptr, flags, out);
}

void msh_free(msh_model* m) { delete m; }

int msh_get_scalars(const msh_model* m, msh_scalars* o) {
    if (!m || !o) return set_err("null argument");
    const Stuff& s = m->stuff;
    std::memset(o, 0, sizeof(*o));
    o->num_nodes = s.num_nodes;
    o->num_tris = s.num_tris;
    o->num_edges = s.num_edges;
    o->num_boundary_nodes = s.num_boundary_nodes;
    o->num_boundary_edges = s.num_boundary_edges;
    o->dialling_protocol = s.dialling_protocol;
    o->dialling_from_ansatz = s.dialling_from_ansatz_rather_than_ref_state;
    o->using_gradient_descent_dynamics = s.using_gradient_descent_dynamics;
    o->num_gd_steps = s.num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics;
    o->output_regularly = s.output_regularly;
    o->steps_between_outputs = s.steps_between_outputs;
    o->timesteps_per_dial_phase = s.timesteps_per_dial_phase;
    o->timesteps_between_equil_checks = s.timesteps_between_equil_checks;
    o->sample_char_length = s.sample_char_length;
    o->approx_min_tri_size = s.approx_min_tri_size;
    o->min_ref_thickness = s.min_ref_thickness;
    o->min_ref_shear_modulus = s.min_ref_shear_modulus;
    o->char_long_time = s.char_long_time;
    o->dial_phase_time = s.dial_phase_time;
    o->timestep = s.timestep;
    o->damping_factor_1 = m->damping_factor_1;
    o->damping_factor_2 = m->damping_factor_2;
    o->char_force_scale = s.char_force_scale;
    o->char_speed_scale = s.char_speed_scale;
    o->char_stretch_energy_density_scale = s.char_stretch_energy_density_scale;
    o->total_ref_area = s.total_ref_area;
    o->dial_factors_to_hold_at_spacing = s.dial_factors_to_hold_at_spacing;
    o->dial_factor_to_start_from = m->dial_factor_to_start_from;
    o->def_poisson_ratio = s.def_poisson_ratio;
    o->bend_stiffening_scale_factor = s.bend_stiffening_scale_factor;
    o->ref_density = s.ref_density;
    o->force_thresh = s.force_to_char_force_ratio_equil_threshold;
    o->speed_thresh = s.speed_to_char_speed_ratio_equil_threshold;
    return 0;
}

int msh_get_desc(const msh_model* m, ms_mesh_desc* d, ms_params* p) {
    if (!m) return set_err("null argument");
    if (d) {
        d->num_nodes = m->stuff.num_nodes;
        d->num_tris = m->stuff.num_tris;
        d->patch_ids = m->patch_ids.data();
        d->deriv_coeffs = m->coeffs.data();
        d->ref_area = m->area.data();
        d->ref_thickness = m->thick.data();
        d->ref_shear_modulus = m->shear.data();
        d->node_mass = m->mass.data();
        d->is_constrained = m->fixed.data();
        d->is_boundary = m->boundary.data();
    }
    if (p) {
        const Stuff& s = m->stuff;
        p->def_poisson_ratio = s.def_poisson_ratio;
        p->bend_stiffening_scale_factor = s.bend_stiffening_scale_factor;
        p->ref_density = s.ref_density;
        p->min_ref_thickness = s.min_ref_thickness;
        p->char_force_scale = s.char_force_scale;
        p->char_speed_scale = s.char_speed_scale;
        p->force_to_char_force_ratio_equil_threshold = s.force_to_char_force_ratio_equil_threshold;
        p->speed_to_char_speed_ratio_equil_threshold = s.speed_to_char_speed_ratio_equil_threshold;
    }
    return 0;
}

int msh_get_dofs(const msh_model* m, int which, double* dofs) {
    if (!m || !dofs) return set_err("null argument");
    soa_from(which == 0 ? m->ref_positions : m->init_positions, dofs);
    return 0;
}

int msh_get_programmed(const msh_model* m, double* a, int32_t* ka, double* b, int32_t* kb) {
    if (!m) return set_err("null argument");
    if (ka) *ka = m->abar_info.cols;
    if (kb) *kb = m->bbar_info.cols;
    if (a) std::memcpy(a, m->abar_info.v.data(), m->abar_info.v.size() * sizeof(double));
    if (b) std::memcpy(b, m->bbar_info.v.data(), m->bbar_info.v.size() * sizeof(double));
    return 0;
}

int msh_get_tri_vertices(const msh_model* m, int32_t* ids) {
    if (!m || !ids) return set_err("null argument");
    for (size_t t = 0; t < m->tris.size(); ++t)
        for (int v = 0; v < 3; ++v) ids[3 * t + v] = m->tris[t].vertex_ids[v];
    return 0;
}

int msh_get_boundary(const msh_model* m, uint8_t* b) {
    if (!m || !b) return set_err("null argument");
    std::memcpy(b, m->boundary.data(), m->boundary.size());
    return 0;
}

// The dynamics loop, main.cpp:269-508.  Runs of steps that need no host
// decision go to the fused GPU stepper (ms_step_n); steps that check for
// equilibrium or write output go through the one-call-per-function path so
// that the check and the output see the state before the update, as in the
// reference.  With the mixed-precision path a check step is one fused step
// instead, so that equilibrium is judged on the forces that path steps with.
int msh_run(msh_model* model, const msh_run_options* opts, msh_run_result* res, double* dofs_out) {
    if (!model || !opts || !res) return set_err("null argument");
    std::memset(res, 0, sizeof(*res));
    Stuff st = model->stuff;  // per-run copy (status, damping, timestep change)
    Log log;
    log.set_quiet(opts->quiet != 0);
    if (opts->output_dir) {
        std::filesystem::create_directories(opts->output_dir);
        st.output_dir_path = opts->output_dir;
        st.aux_output_filepath = std::string(opts->output_dir) + "/aux_output.txt";
        log.set_output_filepath(std::string(opts->output_dir) + "/log.txt");
    }
    const int N = st.num_nodes, T = st.num_tris;
    auto wall0 = std::chrono::steady_clock::now();

    ms_mesh_desc desc;
    ms_params prm;
    msh_get_desc(model, &desc, &prm);
    ms_handle* h = nullptr;
    int rc = ms_create(&desc, &prm, opts->device, opts->precision, &h);
    if (rc != MS_OK) return set_err(std::string("ms_create failed: ") + ms_status_string(rc));
    std::unique_ptr<ms_handle, decltype(&ms_destroy)> guard(h, &ms_destroy);
    auto gpu = [&](int code, const char* what) {
        if (code != MS_OK)
            throw std::runtime_error(std::string(what) + ": " + ms_status_string(code) + " (" + ms_last_error(h) + ")");
    };

    std::vector<double> dofs(3ULL * N);
    soa_from(model->init_positions, dofs.data());
    double time = 0.0;
    long long stepcount = 0;
    double dial_factor = model->dial_factor_to_start_from;
    long long tsc = -123456;  // timesteps_since_previous_equil_check
    double last_equil_dial = model->dial_factor_to_start_from;
    long long k_phase = static_cast<long long>(std::fmod(model->dial_factor_to_start_from, st.dial_factors_to_hold_at_spacing) *
                                               static_cast<double>(st.timesteps_per_dial_phase));
    st.status = dialling;
    st.damping_factor = model->damping_factor_1;
    const bool gd_at_start = st.using_gradient_descent_dynamics;
    const int gd_steps = st.num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics;
    std::vector<double> dials;
    std::vector<double> curv(2ULL * T), edens(2ULL * T), strains(T), stresses(8ULL * T), deficits(N);
    double energies[3];
    int code = MS_OK;
    log << std::scientific << std::setprecision(8);
    try {
        gpu(ms_upload_dofs(h, dofs.data(), nullptr), "ms_upload_dofs");
        gpu(ms_set_programmed(h, st.dialling_protocol, model->abar_info.v.data(), model->abar_info.cols,
                              model->bbar_info.v.data(), model->bbar_info.cols, st.dial_factors_to_hold_at_spacing,
                              st.dialling_from_ansatz_rather_than_ref_state),
            "ms_set_programmed");
        log << "Beginning dynamics loop." << std::endl;

        // Output quantities of the current state, then the files.
        auto snap_out = [&]() {
            gpu(ms_output_quantities(h, curv.data(), edens.data(), strains.data(), stresses.data(), deficits.data(),
                                     energies),
                "ms_output_quantities");
            gpu(ms_download_dofs(h, dofs.data(), nullptr), "ms_download_dofs");
        };
        auto emit_out = [&](long long step) {
            if (opts->write_outputs && opts->output_dir)
                write_output(dofs, model->tris, (int)step, dial_factor, curv, edens, deficits, stresses, strains, st);
        };
        auto write_out = [&](long long step) {
            snap_out();
            emit_out(step);
        };
        auto log_check = [&](const ms_equil_result& eq) {
            res->last_max_force_ratio = eq.max_force / st.char_force_scale;
            res->last_max_speed_ratio = eq.max_speed / st.char_speed_scale;
            log << "Max ratio of non-damping force to characteristic force = " << res->last_max_force_ratio
                << " (node " << eq.max_force_node << ")" << "\n";
            log << "Max ratio of node speed to characteristic speed = " << res->last_max_speed_ratio << " (node "
                << eq.max_speed_node << ")" << "\n";
            if (eq.at_equilibrium) {
                st.status = equil_reached;
                res->equilibria_reached += 1;
                log << "Equilibrium reached. Writing VTK output at " << get_real_time() << ", stepcount = "
                    << stepcount << ", simulation time = " << time << ", dial_factor = " << dial_factor << std::endl;
                last_equil_dial = dial_factor;
            }
            tsc = 0;
        };
        auto crash = [&](long long dof, double force) {
            log << " ------------CRASH REPORT-----------------" << std::endl;
            log << "Offending dof is " << dof << std::endl;
            log << "Offending force is " << force << std::endl;
            log << "Offending node is " << dof % N << std::endl;
            write_out(stepcount);
            log << "At stepcount = " << stepcount << ", dial_factor = " << dial_factor
                << " there was a problem: implausibly_high_force" << std::endl;
        };

        for (;;) {
            if (opts->max_steps > 0 && stepcount >= opts->max_steps) break;
            // main.cpp:273-279
            if (st.using_gradient_descent_dynamics && stepcount > gd_steps) {
                log << "Finished doing gradient descent, now switching to Newtonian dynamics." << std::endl;
                st.using_gradient_descent_dynamics = false;
                calc_steps_between_outputs(st, log);
                calc_timestep(st, log);
            }
            if (dial_factor >= 1.0) dial_factor = 1.0;  // :286-288
            if (st.status == dialling && k_phase >= st.timesteps_per_dial_phase) {  // :293-304
                st.status = waiting_for_equil;
                tsc = 0;
                st.damping_factor = model->damping_factor_2;
                calc_timestep(st, log);
                log << "Reached dial_factor = " << dial_factor << ", now waiting for equilibrium." << std::endl;
            }
            const bool check = st.status == waiting_for_equil && tsc > st.timesteps_between_equil_checks;
            const bool regular_out = st.output_regularly && st.steps_between_outputs > 0 &&
                                     (stepcount % st.steps_between_outputs == 0) && opts->write_outputs;
            const bool host_step = stepcount == 0 || check || regular_out;
            if (!host_step) {
                // Fuse the run of plain steps that starts here.  Simulate the
                // scalar state machine to find where it ends.
                long long room = opts->max_steps > 0 ? opts->max_steps - stepcount : (1LL << 40);
                const bool dialling_now = st.status == dialling;
                const bool gd = st.using_gradient_descent_dynamics;
                dials.clear();
                long long n = 0;
                double df = dial_factor;
                long long k = k_phase, ts = tsc, sc = stepcount;
                for (;;) {
                    if (n >= room || n >= 1 << 20) break;
                    if (gd && sc > gd_steps) break;
                    if (df >= 1.0) df = 1.0;
                    if (dialling_now && k >= st.timesteps_per_dial_phase) break;
                    if (!dialling_now && ts > st.timesteps_between_equil_checks) break;
                    if (st.output_regularly && st.steps_between_outputs > 0 && sc % st.steps_between_outputs == 0 &&
                        opts->write_outputs)
                        break;
                    if (dialling_now) dials.push_back(df);
                    ++n;
                    ++sc;
                    if (dialling_now) ++k;
                    df = last_equil_dial + st.dial_factors_to_hold_at_spacing *
                                               (static_cast<double>(k) / static_cast<double>(st.timesteps_per_dial_phase));
                    if (!dialling_now) ++ts;
                }
                if (n > 0) {
                    ms_step_report rep;
                    code = ms_step_n(h, (int)n, dialling_now ? dials.data() : nullptr, dialling_now ? 1 : 0, st.timestep,
                                     st.damping_factor, gd ? 1 : 0, 0, &rep);
                    if (code == MS_ERR_IMPLAUSIBLE_FORCE) {
                        // Advance the scalar state to the failing step, then
                        // report and dump as main.cpp:448-474 does.
                        for (int i = 0; i < rep.steps_done; ++i) {
                            time += st.timestep;
                            ++stepcount;
                            if (dialling_now) ++k_phase;
                            dial_factor = last_equil_dial + st.dial_factors_to_hold_at_spacing *
                                                                (static_cast<double>(k_phase) /
                                                                 static_cast<double>(st.timesteps_per_dial_phase));
                            if (!dialling_now) ++tsc;
                        }
                        if (dialling_now) dial_factor = dials[rep.steps_done];
                        crash(rep.offending_dof, rep.offending_force);
                        break;
                    }
                    gpu(code, "ms_step_n");
                    for (long long i = 0; i < n; ++i) {
                        time += st.timestep;
                        ++stepcount;
                        if (dialling_now) ++k_phase;
                        dial_factor = last_equil_dial + st.dial_factors_to_hold_at_spacing *
                                                            (static_cast<double>(k_phase) /
                                                             static_cast<double>(st.timesteps_per_dial_phase));
                        if (!dialling_now) ++tsc;
                    }
                    continue;
                }
            }
            if (check && opts->precision == MS_PRECISION_MIXED) {
                // The mixed-precision path judges equilibrium in its own
                // force field (float per-triangle arithmetic, double node
                // sums): one fused step that also reduces |F| and |v| of
                // the state before its update (is_at_equilibrium.cpp:62-84).
                const bool outputs = opts->write_outputs && opts->output_dir;
                if (outputs) snap_out();
                log << "Checking for equilibrium at " << get_real_time() << ", stepcount = " << stepcount
                    << ", simulation time = " << time << ", dial_factor = " << dial_factor << std::endl;
                ms_step_report rep;
                code = ms_step_n(h, 1, nullptr, 0, st.timestep, st.damping_factor,
                                 st.using_gradient_descent_dynamics ? 1 : 0, 1, &rep);
                if (code == MS_ERR_IMPLAUSIBLE_FORCE) {
                    crash(rep.offending_dof, rep.offending_force);
                    break;
                }
                gpu(code, "ms_step_n");
                log_check(rep.equil);
                if (outputs && (regular_out || st.status == equil_reached)) emit_out(stepcount);
            } else {
                // One step through the per-function path (main.cpp:308-474).
                gpu(ms_surface_derivs(h, nullptr), "calc_surface_derivs");
                if (stepcount == 0 && st.dialling_from_ansatz_rather_than_ref_state) {
                    std::vector<double> a(3ULL * T), b(3ULL * T), nn(3ULL * T);
                    gpu(ms_a_b_normals(h, a.data(), b.data(), nn.data()), "calc_a_comps_and_b_comps_and_normals");
                    gpu(ms_set_zero_dial_state(h, a.data(), b.data()), "ms_set_zero_dial_state");
                }
                if (st.status == dialling || stepcount == 0) gpu(ms_do_dialling(h, dial_factor), "do_dialling");
                gpu(ms_deformation_forces(h, nullptr, nullptr), "calc_deformation_forces");
                gpu(ms_non_deformation_forces(h, st.damping_factor, st.using_gradient_descent_dynamics),
                    "calc_non_deformation_forces");
                gpu(ms_impose_constraints(h), "impose_constraints");
                if (check) {
                    log << "Checking for equilibrium at " << get_real_time() << ", stepcount = " << stepcount
                        << ", simulation time = " << time << ", dial_factor = " << dial_factor << std::endl;
                    ms_equil_result eq;
                    gpu(ms_is_at_equilibrium(h, &eq), "is_at_equilibrium");
                    log_check(eq);
                }
                if (regular_out || st.status == equil_reached) {
                    if (opts->write_outputs) write_out(stepcount);
                }
                int64_t bad_dof = -1;
                double bad_force = 0.0;
                code = ms_advance_dynamics(h, st.timestep, st.damping_factor, st.using_gradient_descent_dynamics,
                                           &bad_dof, &bad_force);
                if (code == MS_ERR_IMPLAUSIBLE_FORCE) {
                    crash(bad_dof, bad_force);
                    break;
                }
                gpu(code, "advance_dynamics");
            }
            time += st.timestep;
            stepcount += 1;
            if (st.status == dialling) k_phase += 1;
            dial_factor = last_equil_dial + st.dial_factors_to_hold_at_spacing *
                                                (static_cast<double>(k_phase) / static_cast<double>(st.timesteps_per_dial_phase));
            if (st.status == waiting_for_equil) tsc += 1;
            // The reference leaves the loop only when glass slides are on
            // (main.cpp:493-495); the option below stops at the first
            // equilibrium reached at full dial factor instead.
            if (st.status == equil_reached && last_equil_dial >= 1.0 && opts->stop_at_final_equilibrium) {
                res->final_status = st.status;
                dial_factor = last_equil_dial;  // report the dial factor equilibrium was reached at
                break;
            }
            if (st.status == equil_reached) {  // :501-507
                st.status = dialling;
                k_phase = 0;
                st.damping_factor = model->damping_factor_1;
                calc_timestep(st, log);
            }
        }
        log << "Simulation completed at time = " << time << ", stepcount = " << stepcount << std::endl;
        if (dofs_out) gpu(ms_download_dofs(h, dofs_out, nullptr), "ms_download_dofs");
    } catch (const std::exception& e) {
        res->status = MS_ERR_CUDA;
        return set_err(e.what());
    }
    (void)gd_at_start;
    res->status = code;
    res->steps = stepcount;
    res->final_dial_factor = dial_factor;
    res->sim_time = time;
    if (res->final_status == 0) res->final_status = st.status;
    res->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    return code == MS_OK ? 0 : set_err("implausibly_high_force");
}

// Many models through one ms_batch: each keeps the state machine of
// msh_run (main.cpp:269-508) on the device.  Supports what the batch
// supports: protocol 3 without ansatz dialling, Newtonian dynamics, no
// regular output.
int msh_run_batch(msh_model* const* models, int32_t n, const msh_run_options* opts, msh_run_result* results,
                  double* const* dofs_out) {
    if (!models || n <= 0 || !opts || !results) return set_err("null argument");
    if (opts->max_steps <= 0 && !opts->stop_at_final_equilibrium)
        return set_err("msh_run_batch needs max_steps > 0 or stop_at_final_equilibrium");
    auto wall0 = std::chrono::steady_clock::now();
    std::vector<ms_batch_instance> inst(n);
    std::vector<std::vector<double>> info(n), dofs(n);
    for (int i = 0; i < n; ++i) {
        msh_model* m = models[i];
        if (!m) return set_err("null model");
        const Stuff& st = m->stuff;
        if (st.dialling_protocol != 3 || st.dialling_from_ansatz_rather_than_ref_state || m->abar_info.cols < 3)
            return set_err("msh_run_batch: model " + std::to_string(i) +
                           " is not protocol-3 dialling from the reference state");
        if (st.using_gradient_descent_dynamics)
            return set_err("msh_run_batch: model " + std::to_string(i) + " uses gradient-descent steps");
        const int T = st.num_tris, N = st.num_nodes;
        info[i].resize(3ULL * T);
        for (int t = 0; t < T; ++t)
            for (int k = 0; k < 3; ++k) info[i][3ULL * t + k] = m->abar_info(t, k);
        dofs[i].resize(3ULL * N);
        soa_from(m->init_positions, dofs[i].data());
        ms_batch_instance& b = inst[i];
        std::memset(&b, 0, sizeof(b));
        msh_get_desc(m, &b.mesh, &b.params);
        b.abar_info = info[i].data();
        b.timestep = st.timestep;
        b.damping_factor_1 = m->damping_factor_1;
        b.damping_factor_2 = m->damping_factor_2;
        b.timesteps_per_dial_phase = st.timesteps_per_dial_phase;
        b.timesteps_between_equil_checks = st.timesteps_between_equil_checks;
        b.dial_factors_to_hold_at_spacing = st.dial_factors_to_hold_at_spacing;
        b.dial_factor_to_start_from = m->dial_factor_to_start_from;
        b.stop_at_final_equilibrium = opts->stop_at_final_equilibrium ? 1 : 0;
        b.dofs = dofs[i].data();
        b.velocities = nullptr;
    }
    ms_batch* batch = nullptr;
    int rc = ms_batch_create(inst.data(), n, opts->device, opts->precision, &batch);
    if (rc != MS_OK) return set_err(std::string("ms_batch_create failed: ") + ms_status_string(rc));
    std::unique_ptr<ms_batch, decltype(&ms_batch_destroy)> guard(batch, &ms_batch_destroy);
    int64_t done = 0;
    rc = ms_batch_run(batch, opts->max_steps > 0 ? opts->max_steps : INT64_MAX / 2, &done);
    if (rc != MS_OK) return set_err(std::string("ms_batch_run: ") + ms_batch_last_error(batch));
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    for (int i = 0; i < n; ++i) {
        ms_batch_inst_status bs;
        rc = ms_batch_status(batch, i, &bs);
        if (rc != MS_OK) return set_err(std::string("ms_batch_status: ") + ms_batch_last_error(batch));
        msh_run_result& r = results[i];
        std::memset(&r, 0, sizeof(r));
        r.status = bs.status == MS_INST_FAILED ? MS_ERR_IMPLAUSIBLE_FORCE : MS_OK;
        r.steps = bs.stepcount;
        r.final_dial_factor = bs.dial_factor;
        r.sim_time = bs.sim_time;
        r.equilibria_reached = bs.equilibria;
        r.final_status = bs.status == MS_INST_DONE      ? equil_reached
                         : bs.status == MS_INST_WAITING ? waiting_for_equil
                                                        : dialling;
        r.wall_seconds = wall;
        r.last_max_force_ratio = bs.max_force_ratio;
        r.last_max_speed_ratio = bs.max_speed_ratio;
        if (dofs_out && dofs_out[i]) {
            rc = ms_batch_download_dofs(batch, i, dofs_out[i], nullptr);
            if (rc != MS_OK) return set_err(std::string("ms_batch_download_dofs: ") + ms_batch_last_error(batch));
        }
    }
    return 0;
}

}  // extern "C"
