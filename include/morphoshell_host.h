/*
 * morphoshell_host.h -- C ABI of the host-side set-up and main-loop driver.
 *
 * msh_load runs the reference's one-off set-up sequence (main.cpp:74-238):
 * read_settings, read_vtk_data, calc_mesh_info, set_up_patch_fitting,
 * calc_deriv_mats, calc_dof_masses, the characteristic scales, timestep and
 * dialling schedule, perturb_node_positions_with_noise and the ansatz move.
 * msh_get_desc hands its tables to ms_create (morphoshell_gpu.h).  msh_run
 * drives the dynamics loop of main.cpp:269-508 on the GPU.
 *
 * Errors: functions return 0 on success; otherwise msh_last_error() holds
 * the reference's std::runtime_error message for the calling thread.
 */
#ifndef MORPHOSHELL_HOST_H
#define MORPHOSHELL_HOST_H

#include <stdint.h>

#include "morphoshell_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct msh_model msh_model;

/* Derived scalars of Stuff_Class after set-up. */
typedef struct msh_scalars {
    int32_t num_nodes, num_tris, num_edges, num_boundary_nodes, num_boundary_edges;
    int32_t dialling_protocol;
    int32_t dialling_from_ansatz;
    int32_t using_gradient_descent_dynamics;
    int32_t num_gd_steps;
    int32_t output_regularly;
    int64_t steps_between_outputs;
    int64_t timesteps_per_dial_phase;
    int64_t timesteps_between_equil_checks;
    double sample_char_length, approx_min_tri_size, min_ref_thickness, min_ref_shear_modulus;
    double char_long_time, dial_phase_time, timestep;
    double damping_factor_1, damping_factor_2;  /* damping_factor for prefactors 1 and 2 */
    double char_force_scale, char_speed_scale, char_stretch_energy_density_scale, total_ref_area;
    double dial_factors_to_hold_at_spacing, dial_factor_to_start_from;
    double def_poisson_ratio, bend_stiffening_scale_factor, ref_density;
    double force_thresh, speed_thresh;
} msh_scalars;

/* settings_path and vtk_path as the reference's command line; ansatz_path
 * may be NULL.  flags: bit 0 quiet (no stdout), bit 1 skip the initial noise,
 * bit 2 patch search, patch fit and derivative weights on the current CUDA
 * device (the host's results, bit for bit; triangles whose candidate
 * distances tie are redone on the host). */
int msh_load(const char* settings_path, const char* vtk_path, const char* ansatz_path, int flags, msh_model** out);
/* Same set-up with the mesh handed over in memory instead of a VTK file
 * (the CELL_DATA / POINT_DATA fields of read_vtk_data.cpp as arrays):
 * positions N x 3, tri_vertex_ids T x 3, abar_info T x ka, bbar_info T x kb,
 * all row-major; ref_thicknesses / ref_shear_moduli (T) may be NULL when the
 * settings give uniform values; constrained (N) may be NULL. */
int msh_build(const char* settings_path, int32_t num_nodes, int32_t num_tris, const double* positions,
              const int32_t* tri_vertex_ids, const double* abar_info, int32_t ka, const double* bbar_info, int32_t kb,
              const double* ref_thicknesses, const double* ref_shear_moduli, const uint8_t* constrained, int flags,
              msh_model** out);
void msh_free(msh_model* m);
const char* msh_last_error(void);

int msh_get_scalars(const msh_model* m, msh_scalars* out);
/* Pointers stay valid until msh_free. */
int msh_get_desc(const msh_model* m, ms_mesh_desc* desc, ms_params* params);
/* which: 0 reference (flat) positions, 1 initial dofs of the dynamics (after
 * noise and any ansatz).  dofs is SoA [X(N) | Y(N) | Z(N)]. */
int msh_get_dofs(const msh_model* m, int which, double* dofs);
/* abar_info / bbar_info (num_tris x k, row-major); pass NULL to query k. */
int msh_get_programmed(const msh_model* m, double* abar_info, int32_t* ka, double* bbar_info, int32_t* kb);
/* Triangle vertex ids (3T) and patch data, for tests. */
int msh_get_tri_vertices(const msh_model* m, int32_t* ids);
int msh_get_boundary(const msh_model* m, uint8_t* is_boundary);

typedef struct msh_run_options {
    int64_t max_steps;          /* stop after this many steps (<= 0: no limit) */
    int32_t stop_at_final_equilibrium; /* stop at the first equilibrium with dial_factor >= 1 */
    int32_t write_outputs;      /* write VTK output files as the reference does */
    int32_t precision;          /* ms_precision */
    int32_t device;
    int32_t quiet;
    const char* output_dir;     /* directory for output files and the log (NULL: no files) */
} msh_run_options;

typedef struct msh_run_result {
    int32_t status;             /* ms_status of the run */
    int64_t steps;              /* steps advanced */
    double final_dial_factor;
    double sim_time;
    int32_t equilibria_reached;
    int32_t final_status;       /* Status_Enum */
    double wall_seconds;
    double last_max_force_ratio, last_max_speed_ratio;
} msh_run_result;

/* Runs the dynamics loop; dofs_out (3N, may be NULL) receives the final state. */
int msh_run(msh_model* m, const msh_run_options* opts, msh_run_result* res, double* dofs_out);

/* Runs n models together as one batch (ms_batch_*): every model follows
 * msh_run's loop independently; max_steps bounds the batch's steps.  No
 * reference counterpart (the reference runs one mesh per process).  Needs
 * protocol-3 dialling from the reference state and Newtonian dynamics;
 * write_outputs and output_dir are ignored.  results[i] and dofs_out[i]
 * (3N_i or NULL; dofs_out itself may be NULL) receive each model's outcome. */
int msh_run_batch(msh_model* const* models, int32_t n, const msh_run_options* opts, msh_run_result* results,
                  double* const* dofs_out);

#ifdef __cplusplus
}
#endif

#endif /* MORPHOSHELL_HOST_H */
