// Host-side data model and set-up of the MorphoShell force-and-dynamics loop.
//
// These are the reference's own entry points (same names, same argument
// meaning, same std::runtime_error convention) re-expressed over plain
// std::vector storage instead of Eigen objects, which the GPU path never
// sees.  Each function cites the reference file it follows.  The per-step
// physics does not live here: it runs on the GPU behind the C ABI declared in
// include/morphoshell_gpu.h.
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace msb {

// Threads for the host set-up's loops over n items: MORPHOSHELL_SETUP_THREADS,
// else the hardware's; one for small inputs.
inline int setup_threads(long long n) {
    if (n < 4096) return 1;
    int t = (int)std::thread::hardware_concurrency();
    if (const char* e = std::getenv("MORPHOSHELL_SETUP_THREADS")) t = std::atoi(e);
    return std::max(1, std::min(t, 128));
}

// f(begin, end, worker) over [0, n) in contiguous ranges, one per thread.
// The first exception (of the lowest range) is rethrown after all joined.
template <typename F>
void parallel_ranges(int n, int threads, F f) {
    threads = std::max(1, std::min(threads, std::max(n, 1)));
    if (threads <= 1) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> pool;
    std::vector<std::exception_ptr> errs(threads);
    const int chunk = (n + threads - 1) / threads;
    for (int w = 0; w < threads; ++w)
        pool.emplace_back([&, w]() {
            try {
                f(std::min(n, w * chunk), std::min(n, (w + 1) * chunk), w);
            } catch (...) {
                errs[w] = std::current_exception();
            }
        });
    for (auto& t : pool) t.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

// source_files/Status_Enum.hpp:29
enum Status_Enum { dialling, waiting_for_equil, equil_reached };

// Settings and run-time scalars; same members and meaning as
// source_files/Stuff_Class.hpp:34-118.
struct Stuff {
    // Read from the settings file, in file order (read_settings.cpp:90-188).
    double outputs_per_char_long_time = 0;
    double ref_thickness_if_uniform = 0;
    double timestep_prefactor = 0;
    bool dialling_from_ansatz_rather_than_ref_state = false;
    double dial_factors_to_hold_at_spacing = 0;
    double dial_phase_time_prefactor = 0;
    double time_between_equil_checks_prefactor = 0;
    double damping_prefactor_1 = 0;
    double damping_prefactor_2 = 0;
    int num_steps_to_use_gradient_descent_dynamics_for_before_switching_to_newtonian_dynamics = 0;
    double force_to_char_force_ratio_equil_threshold = 0;
    double speed_to_char_speed_ratio_equil_threshold = 0;
    double def_poisson_ratio = 0;
    double ref_shear_modulus_if_uniform = 0;
    double ref_density = 0;
    double bend_stiffening_scale_factor = 0;
    double patch_mat_dimless_conditioning_thresh = 0;
    double slide_stiffness_prefactor = 0;
    double slide_friction_coefficent = 0;
    double slide_speed_prefactor = 0;
    bool using_initial_glass_slide_z_coords_from_settings_file = false;
    double initial_upper_slide_z_coord = 0;
    double initial_lower_slide_z_coord = 0;
    // Optional trailing setting (not in the reference's file format): which
    // dialling protocol of do_dialling.cpp to run.  The reference selects it
    // by editing source; 1 is its shipped default.
    int dialling_protocol = 1;

    // Computed at run time.
    std::string settings_filepath, ref_data_filepath, ansatz_filepath, output_dir_path, aux_output_filepath;
    bool ansatz_file_was_given = false;
    bool output_regularly = false;
    double sample_char_length = 0, approx_min_tri_size = 0, min_ref_thickness = 0, min_ref_shear_modulus = 0;
    double stretch_long_time = 0, bend_long_time = 0, char_long_time = 0, dial_phase_time = 0;
    long timesteps_between_equil_checks = 0;
    double damping_factor = 0, timestep = 0;
    long steps_between_outputs = 0;
    double char_flexural_rigidity = 0, char_force_scale = 0, char_speed_scale = 0;
    double char_stretch_energy_density_scale = 0, char_stretch_energy_scale = 0, total_ref_area = 0;
    double upper_slide_z_coord = 0, upper_slide_tot_vert_force = 0, lower_slide_z_coord = 0, lower_slide_tot_vert_force = 0;
    bool using_gradient_descent_dynamics = false;
    long timesteps_per_dial_phase = 0;
    Status_Enum status = dialling;
    int num_nodes = 0, num_boundary_nodes = 0, num_tris = 0, num_boundary_tris = 0, num_edges = 0,
        num_boundary_edges = 0, num_dofs = 0, num_continuum_quantities = 0;
};

// Per-triangle members the loop uses (source_files/Tri_Class.hpp:40-164).
struct Tri {
    int id = -1;
    bool tag = false;
    bool is_boundary = false;
    std::array<int, 3> vertex_ids{};
    std::array<int, 3> edge_ids{};
    std::array<int, 3> non_vertex_patch_nodes_ids{};
    std::vector<int> edge_sharing_tri_ids;
    double ref_centroid[3] = {0, 0, 0};
    double mat_for_patch_2nd_derivs[6][3] = {};
    double ref_area = 0, ref_thickness = 0, ref_shear_modulus = 0;
};

// source_files/Node_Class.hpp:39-60
struct Node {
    int id = -1;
    std::vector<int> incident_tri_ids;
    std::vector<int> neighbour_node_ids;
    bool is_boundary = false;
    bool tag = false;
    bool is_constrained = false;
};

// source_files/Edge_Class.hpp
struct Edge {
    int id = -1;
    std::array<int, 2> node_ids{};
    std::vector<int> adjacent_tri_ids;
    bool is_boundary = false;
};

// Row-major dense matrix of doubles.
struct DMat {
    int rows = 0, cols = 0;
    std::vector<double> v;
    void resize(int r, int c) { rows = r; cols = c; v.assign(static_cast<size_t>(r) * c, 0.0); }
    double& operator()(int i, int j) { return v[static_cast<size_t>(i) * cols + j]; }
    double operator()(int i, int j) const { return v[static_cast<size_t>(i) * cols + j]; }
};

// Tee logger (source_files/Out_Stream_Class.hpp:76-89).  The reference opens
// and closes its file on every <<; this one keeps the file open.
class Log {
public:
    void set_output_filepath(const std::string& p) {
        path_ = p;
        if (file_.is_open()) file_.close();
        if (!p.empty()) {
            file_.open(p, std::ofstream::app);
            if (!file_) throw std::runtime_error("Error: Problem creating or opening output_filestream.");
        }
    }
    const std::string& get_output_filepath() const { return path_; }
    void set_quiet(bool q) { quiet_ = q; }
    template <typename T>
    Log& operator<<(const T& x) {
        if (!quiet_) std::cout << x;
        if (file_.is_open()) file_ << x;
        return *this;
    }
    typedef std::ostream& (*stream_function)(std::ostream&);
    Log& operator<<(stream_function f) {
        if (!quiet_) f(std::cout);
        if (file_.is_open()) f(file_);
        return *this;
    }

private:
    std::string path_;
    std::ofstream file_;
    bool quiet_ = false;
};

// ---- set-up (once per run) ----------------------------------------------
void read_settings(Stuff& stuff, Log& log);                                   // read_settings.cpp:47
void read_vtk_data(std::vector<Node>& nodes, DMat& node_positions,            // read_vtk_data.cpp:65
                   std::vector<std::array<double, 3>>& ansatz_node_positions,
                   std::vector<Tri>& triangles, DMat& abar_info, DMat& bbar_info,
                   Stuff& stuff, double& dial_factor_to_start_from, Log& log);
void calc_mesh_info(std::vector<Node>& nodes, const DMat& node_positions,     // calc_mesh_info.cpp:50
                    std::vector<Tri>& triangles, std::vector<Edge>& edges, Stuff& stuff, Log& log);
void set_up_patch_fitting(const std::vector<Node>& nodes, const DMat& node_positions,  // set_up_patch_fitting.cpp:48
                          std::vector<Tri>& triangles, const Stuff& stuff, Log& log);
// calc_deriv_mats.cpp:46, stored densely: 24 coefficients per triangle,
// [d/dx of vertices 0..2, d/dy of vertices 0..2, then for patch node n=0..5
// the (xx, xy, yy) second-derivative weights].
void calc_deriv_coeffs(std::vector<double>& coeffs, const DMat& node_positions,
                       const std::vector<Tri>& triangles, const Stuff& stuff);
// One triangle's patch search and fit (the loop body of set_up_patch_fitting;
// throws as it does), its 24 weights (calc_deriv_coeffs for one triangle) and
// the set-up's retry report.
void fit_patch(int t_index, const std::vector<Node>& nodes, const DMat& node_positions, std::vector<Tri>& triangles,
               double thresh, int& num_interior_retries);
void deriv_coeffs_of(const Tri& tri, const DMat& node_positions, double* coeffs24);
void log_patch_retries(Log& log, int num_interior_retries);
// set_up_patch_fitting and calc_deriv_coeffs on the current CUDA device
// (setup.cu), with the same results: triangles whose candidate distances tie
// (where the order std::sort gives them is the host's to decide) or whose
// search the device cannot finish are redone on the host.
void set_up_patches_on_device(const std::vector<Node>& nodes, const DMat& node_positions,
                              std::vector<Tri>& triangles, const Stuff& stuff, std::vector<double>& coeffs,
                              Log& log);
void calc_dof_masses(std::vector<double>& dof_masses, const std::vector<Tri>& triangles,  // calc_dof_masses.cpp:45
                     const Stuff& stuff);
void calc_char_mechanics_scales(const std::vector<Tri>& triangles, Stuff& stuff);         // calc_char_mechanics_scales.cpp:45
void calc_long_timescales(Stuff& stuff, Log& log);                                         // calc_long_timescales.cpp:40
void calc_damping_factor(double damping_prefactor, Stuff& stuff, Log& log);               // calc_damping_factor.cpp:42
void calc_timestep(Stuff& stuff, Log& log);                                                // calc_timestep.cpp:41
void calc_steps_between_outputs(Stuff& stuff, Log& log);                                   // calc_steps_between_outputs.cpp:40
void calc_dialling_procedure_params(Stuff& stuff, Log& log);                               // calc_dialling_procedure_params.cpp:52
void perturb_node_positions_with_noise(DMat& node_positions, const Stuff& stuff);          // perturb_node_positions_with_noise.cpp:45
void initialize_glass_slides(const DMat& node_positions, Stuff& stuff);                    // initialize_glass_slides.cpp:27
double kahan_sum(const std::vector<double>& vec);                                          // kahan_sum.cpp:32

// ---- output --------------------------------------------------------------
// write_output.cpp:46 (VTK layout :77-170, aux file :60-69).  dofs is SoA
// [X(N) | Y(N) | Z(N)].
void write_output(const std::vector<double>& dofs, const std::vector<Tri>& triangles, int stepcount,
                  double dial_factor, const std::vector<double>& curvatures /*T x 2*/,
                  const std::vector<double>& energy_densities /*T x 2*/,
                  const std::vector<double>& angle_deficits /*N*/, const std::vector<double>& stresses /*T x 8*/,
                  const std::vector<double>& strains /*T*/, const Stuff& stuff);

std::string get_real_time();

}  // namespace msb
