/*
 * morphoshell_gpu.h -- C ABI of the B200 force-and-dynamics loop.
 *
 * Drop-in replacement for the per-step functions that MorphoShell's main
 * loop (source_files/main.cpp:269-508) calls with caller-owned Eigen
 * objects.  Here the library owns device memory; host arrays are copied in
 * and out and no host pointer is retained after a call returns.  All arrays
 * are plain C arrays:
 *
 *   dofs, velocities, forces : SoA, [X(N) | Y(N) | Z(N)]      (main.cpp:235-237)
 *   continuum quantities     : 15 per triangle, ordered
 *                              Xx Xy Xxx Xxy Xyy  Yx Yy Yxx Yxy Yyy  Zx Zy Zxx Zxy Zyy
 *                                                               (calc_deriv_mats.cpp:60-61)
 *   a, b, abar, bbar, normals: 3 per triangle (xx, xy, yy) / (x, y, z), row-major
 *
 * Every function returns an ms_status; 0 is success.  One handle belongs to
 * one host thread and one CUDA stream; calls on a handle are not re-entrant.
 * Floating-point work is IEEE double unless the handle was created with
 * MS_PRECISION_MIXED.
 */
#ifndef MORPHOSHELL_GPU_H
#define MORPHOSHELL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ms_status {
    MS_OK = 0,
    MS_ERR_INVALID_ARGUMENT = 1,
    MS_ERR_CUDA = 2,
    MS_ERR_IMPLAUSIBLE_FORCE = 3, /* advance_dynamics.cpp:58-73 ("implausibly_high_force") */
    MS_ERR_NON_FINITE = 4,
    MS_ERR_TIMEOUT = 5,
    MS_ERR_NO_DEVICE = 6,
    MS_ERR_OUT_OF_MEMORY = 7,
    MS_ERR_UNSUPPORTED = 8
} ms_status;

typedef enum ms_precision {
    MS_PRECISION_FP64 = 0,  /* all per-step arithmetic in double */
    MS_PRECISION_MIXED = 1  /* per-triangle arithmetic and gathers in float; node state, metric
                               inverse and reductions in double */
} ms_precision;

/* Mesh tables produced by the host set-up (read_vtk_data, calc_mesh_info,
 * set_up_patch_fitting, calc_deriv_mats, calc_dof_masses).  Triangle t's
 * patch is patch_ids[6t..6t+5]: its three vertices (Tri_Class::vertex_ids)
 * then the three extra patch nodes (Tri_Class::non_vertex_patch_nodes_ids).
 * deriv_coeffs[24t..24t+23] holds the non-zeros of triangle t's 15 rows of
 * the sparse matrix built by calc_deriv_mats.cpp:46-136: d/dx weights of the
 * three vertices, d/dy weights of the three vertices, then for each patch
 * node n = 0..5 its (xx, xy, yy) second-derivative weights. */
typedef struct ms_mesh_desc {
    int32_t num_nodes;
    int32_t num_tris;
    const int32_t* patch_ids;         /* 6 * num_tris */
    const double* deriv_coeffs;       /* 24 * num_tris */
    const double* ref_area;           /* num_tris  (Tri_Class::ref_area) */
    const double* ref_thickness;      /* num_tris  (Tri_Class::ref_thickness) */
    const double* ref_shear_modulus;  /* num_tris  (Tri_Class::ref_shear_modulus) */
    const double* node_mass;          /* num_nodes (dof mass, equal for x, y, z; calc_dof_masses.cpp:50-58) */
    const uint8_t* is_constrained;    /* num_nodes (Node_Class::is_constrained) */
    const uint8_t* is_boundary;       /* num_nodes (Node_Class::is_boundary); may be NULL, used only by
                                         the angle deficits of ms_output_quantities */
} ms_mesh_desc;

/* Scalars of Stuff_Class that the per-step functions read. */
typedef struct ms_params {
    double def_poisson_ratio;
    double bend_stiffening_scale_factor;
    double ref_density;
    double min_ref_thickness;
    double char_force_scale;
    double char_speed_scale;
    double force_to_char_force_ratio_equil_threshold;
    double speed_to_char_speed_ratio_equil_threshold;
} ms_params;

/* Result of is_at_equilibrium (is_at_equilibrium.cpp:51-99). */
typedef struct ms_equil_result {
    double max_force;      /* max over nodes of |F_n| */
    double max_speed;      /* max over nodes of |v_n| */
    int64_t max_force_node;/* first node attaining it */
    int64_t max_speed_node;
    int32_t at_equilibrium;
} ms_equil_result;

/* What the fused stepper did (ms_step_n). */
typedef struct ms_step_report {
    int32_t steps_done;          /* steps fully advanced */
    int32_t error_step;          /* index of the step that failed, or -1 */
    int64_t offending_dof;       /* first dof failing the force guard, or -1 */
    double offending_force;
    ms_equil_result equil;       /* filled when the last step carried an equilibrium check */
} ms_step_report;

typedef struct ms_handle ms_handle;

/* ---- lifetime ------------------------------------------------------- */
/* Uploads the mesh tables; initial dofs and velocities are zero.  device < 0
 * selects the current device.  Replaces the allocations of main.cpp:240-260. */
ms_status ms_create(const ms_mesh_desc* mesh, const ms_params* params, int device, int precision,
                    ms_handle** out);
ms_status ms_destroy(ms_handle* h);
const char* ms_last_error(const ms_handle* h);
const char* ms_status_string(int status);

/* ---- state transfer (move_nodes_to_ansatz_positions.cpp:31-38, output) --- */
ms_status ms_upload_dofs(ms_handle* h, const double* dofs /*3N*/, const double* velocities /*3N or NULL = zeros*/);
ms_status ms_download_dofs(ms_handle* h, double* dofs /*3N or NULL*/, double* velocities /*3N or NULL*/);
ms_status ms_download_forces(ms_handle* h, double* forces /*3N*/);

/* ---- programmed tensors and dialling (do_dialling.cpp:36-260) ---------- */
/* abar_info is num_tris x ka, bbar_info num_tris x kb (row-major, the
 * CELL_DATA fields of the input file).  protocol selects the dialling
 * protocol of do_dialling.cpp (1: linear abar/bbar, 2: bbar then abar,
 * 3: LCE lambda, 4: piecewise lambda checkpoints, 5: isotropic swelling). */
ms_status ms_set_programmed(ms_handle* h, int protocol, const double* abar_info, int ka, const double* bbar_info,
                            int kb, double dial_factors_to_hold_at_spacing, int dialling_from_ansatz);
/* a and b at zero dial factor (main.cpp:213-219 and :320-329); NULL keeps
 * the flat reference state a = I, b = 0. */
ms_status ms_set_zero_dial_state(ms_handle* h, const double* a0 /*3T or NULL*/, const double* b0 /*3T or NULL*/);
/* do_dialling: sets abar, bbar (thickness and modulus stay at reference). */
ms_status ms_do_dialling(ms_handle* h, double dial_factor);
ms_status ms_download_programmed(ms_handle* h, double* abar /*3T*/, double* bbar /*3T*/);

/* ---- the reference's per-step sequence, one call each ------------------ */
/* calc_surface_derivs.cpp:27-34: cq = D * dofs.  cq may be NULL (kept on device). */
ms_status ms_surface_derivs(ms_handle* h, double* cq /*15T or NULL*/);
/* calc_a_comps_and_b_comps_and_normals.cpp:27-62, from the last cq. */
ms_status ms_a_b_normals(ms_handle* h, double* a /*3T*/, double* b /*3T*/, double* normals /*3T*/);
/* calc_deformation_forces.cpp:40-185, from the last cq: dE/dcq per triangle
 * and forces = -D^T dE/dcq.  Either output may be NULL. */
ms_status ms_deformation_forces(ms_handle* h, double* forces /*3N or NULL*/, double* del_energy_by_del_cq /*15T or NULL*/);
/* calc_non_deformation_forces.cpp:37-57 (damping; no glass slides). */
ms_status ms_non_deformation_forces(ms_handle* h, double damping_factor, int using_gradient_descent);
/* impose_constraints.cpp:48-69 */
ms_status ms_impose_constraints(ms_handle* h);
/* is_at_equilibrium.cpp:51-99 */
ms_status ms_is_at_equilibrium(ms_handle* h, ms_equil_result* out);
/* advance_dynamics.cpp:47-93: force guard, then v += dt F / m, x += dt v.
 * Returns MS_ERR_IMPLAUSIBLE_FORCE (state untouched) if the guard trips. */
ms_status ms_advance_dynamics(ms_handle* h, double timestep, double damping_factor, int using_gradient_descent,
                              int64_t* offending_dof, double* offending_force);

/* Deformation forces (forces = -D^T dE/dcq, as ms_deformation_forces) for
 * callers that cannot allocate device memory: host frameworks that route
 * every device allocation through their own pool (an allocation behind the
 * pool's back breaks its accounting), real-time loops that must not allocate
 * after start-up (cudaMalloc can block for an unbounded time).  No
 * counterpart in the reference (which never touches a GPU).  No handle is needed and nothing is allocated: every pointer is a
 * DEVICE pointer the caller owns -- patch_ids 6T, deriv_coeffs 24T, ref_area,
 * ref_thickness, ref_shear_modulus T, abar and bbar 3T (all in the
 * ms_mesh_desc / row-major layouts above), dofs and forces 3N SoA.  Work
 * space is a static device array inside this library, sized for at most
 * 65,536 nodes and 65,536 triangles (about 11.5 MB that every GPU loading
 * the library keeps until exit); larger meshes return
 * MS_ERR_INVALID_ARGUMENT with the reason in err.  Every call looks up that
 * array's device address in the current context (cudaGetSymbolAddress; the
 * first call on a device also loads the library's device code, so make it
 * before any stream capture).  All calls share the array:
 * calls that overlap on the GPU race, so serialise them.  Runs on `stream`
 * (a cudaStream_t, NULL for the default stream) and returns after the forces
 * are written (it waits for the stream, to check the patch ids).  A CUDA
 * error already pending when it is called is reported as MS_ERR_CUDA and
 * left pending; nothing is launched then.  err (err_len bytes, may be NULL)
 * receives a message. */
ms_status ms_deformation_forces_noalloc(int32_t num_nodes, int32_t num_tris, const int32_t* patch_ids,
                                        const double* deriv_coeffs, const double* ref_area,
                                        const double* ref_thickness, const double* ref_shear_modulus,
                                        const double* abar, const double* bbar, double def_poisson_ratio,
                                        double bend_stiffening_scale_factor, const double* dofs, double* forces,
                                        void* stream, char* err, size_t err_len);

/* ---- fused stepper: the whole main.cpp:308-488 body per step ----------
 * Runs n steps of: surface derivs -> (dialling) -> deformation forces ->
 * damping -> constraints -> (equilibrium check on the last step if
 * check_last) -> force guard -> symplectic Euler, as one kernel per step on
 * the node-tiled path (two on the others, ms_set_step_path) captured in CUDA
 * graphs.  Fused protocol-3 steps dial inside the force kernel; the abar and
 * bbar arrays are brought to the last step's dial factor only when a later
 * call reads them (ms_download_programmed, ms_deformation_forces,
 * ms_output_quantities, non-fused steps).  dial_factors[i] (length n, may be NULL when
 * dialling == 0) is the dial factor step i dials to.  Stops at the first
 * step whose force guard trips and reports it; the state is then the state
 * before that step, as in main.cpp:448-474. */
ms_status ms_step_n(ms_handle* h, int n, const double* dial_factors, int dialling, double timestep,
                    double damping_factor, int using_gradient_descent, int check_last, ms_step_report* report);

/* Builds (captures and instantiates) the CUDA graphs that ms_step_n with
 * the same n, dialling, timestep, damping, gradient-descent and check_last
 * arguments would use from the current state buffer, launching nothing, so
 * that the first such call does not pay for them.  No reference counterpart
 * (it only moves set-up work out of the timed loop). */
ms_status ms_prepare_steps(ms_handle* h, int n, int dialling, double timestep, double damping_factor,
                           int using_gradient_descent, int check_last);

/* ---- output diagnostics (main.cpp:412-436) ------------------------------
 * From the current dofs (recomputes cq).  Any output may be NULL.
 * curvatures T x 2 (Gauss, mean; calc_curvatures.cpp), energy_densities
 * T x 2 (stretch, bend; calc_energy_densities.cpp), strains T
 * (calc_strains.cpp), stresses T x 8 (calc_stresses.cpp), angle_deficits N
 * (calc_angle_deficits.cpp), energies[3] = stretch, bend, kinetic
 * (calc_energies.cpp). */
ms_status ms_output_quantities(ms_handle* h, double* curvatures, double* energy_densities, double* strains,
                               double* stresses, double* angle_deficits, double* energies);

/* Library and device description, for logs. */
ms_status ms_device_info(char* buf, size_t len);

/* The cudaStream_t the handle launches on (as void*), for callers that order
 * or time their own work around it. */
void* ms_stream(ms_handle* h);

/* Which implementation ms_step_n uses: 0 the cluster-tiled step -- each
 * thread-block cluster owns a Morton tile of triangles, keeps their force
 * contributions in distributed shared memory and updates the tile's
 * interior nodes itself; 1 the two-kernel step (per-triangle kernel writes
 * all contributions to HBM, per-node kernel gathers them); 2 the two-kernel
 * step whose per-triangle kernel is persistent and streams its tables
 * through shared memory with bulk asynchronous copies; 3 the node-tiled
 * step -- one kernel: each block takes tiles of consecutive nodes, computes
 * every triangle that touches the tile (border triangles once per tile),
 * sums the tile's forces in shared memory and updates its nodes, so no
 * contribution goes through HBM.  The default is 3 on meshes with at least
 * one node tile per resident block, else 2.  All sum every node's
 * contributions in ascending triangle order, so they give the same bits. */
ms_status ms_set_step_path(ms_handle* h, int path);
/* Tiling of the cluster path: CTAs per cluster, triangles per CTA, number of
 * clusters, number of halo nodes (summed by the second kernel), and the
 * path in use. */
ms_status ms_plan_info(ms_handle* h, int* cluster_size, int* tris_per_cta, int* clusters, int* halo_nodes,
                       int* path);

/* The node-tiled step's plan on this handle: nodes per tile, tiles, chunk
 * records and persistent blocks per launch (all 0 when the path is
 * unavailable). */
ms_status ms_node_tile_plan(ms_handle* h, int* nodes_per_tile, int* tiles, int* chunks, int* blocks);
/* Layout of the node-tiled step (path 3) for a mesh and a tile size, computed
 * on the host alone (no device needed), with the same code and the same
 * bounds checks ms_create runs: node tiles, chunk records (128 triangle
 * slots each), triangles computed per step (a border triangle once per tile
 * it touches), the largest node section and the record stride in bytes,
 * the record bytes copied per step and the shared memory a block needs
 * (of the node-tiled step, and of the warp-specialised one).
 * Returns MS_ERR_INVALID_ARGUMENT for bad arguments or lists that fail the
 * checks. */
typedef struct ms_node_tile_info {
    int tiles;
    int chunks;
    long long tri_tile_pairs;
    long long node_section_max;
    long long record_stride;
    long long bytes_per_step;
    long long shared_bytes;
    long long sliced_entries;   /* largest sliced staging of a chunk (entries per component) */
    long long pipe_shared_bytes; /* shared memory a block of the warp-specialised step needs */
} ms_node_tile_info;
ms_status ms_node_tile_layout(int num_nodes, int num_tris, const int* patch_ids, int nodes_per_tile, int precision,
                              ms_node_tile_info* out);

/* Mean device time of one launch of each fused-step kernel over `reps`
 * steps (CUDA events on the handle's stream; the steps advance the state):
 * the per-triangle kernel (ms_tri) and the per-node kernel (ms_node); on
 * the node-tiled path the one kernel is ms_tri and ms_node is 0. */
ms_status ms_time_kernels(ms_handle* h, int reps, int dialling, double dial_factor, double timestep,
                          double damping_factor, double* ms_tri, double* ms_node);

/* ---- batched ensembles -----------------------------------------------------
 * Many independent meshes of any sizes stepped together on one device.  No
 * reference counterpart: the reference runs one mesh per process, and each
 * instance here runs its own copy of that process's main loop
 * (main.cpp:269-508) on the device -- protocol-3 dialling, the wait for
 * equilibrium with checks every timesteps_between_equil_checks steps
 * (is_at_equilibrium.cpp:51-99), the next dial phase, the force guard
 * (advance_dynamics.cpp:58-75) -- with its own timestep, damping,
 * thresholds and programmed field.  An instance that trips the guard is
 * marked failed and keeps the state from before that step; one that reaches
 * equilibrium at dial factor 1 (with stop_at_final_equilibrium) is done;
 * either way it stops while the others go on.  Steps run in chunks captured
 * as CUDA graphs; the host looks at the instance states between chunks. */
typedef struct ms_batch ms_batch;

enum ms_inst_status {
    MS_INST_DIALLING = 0,
    MS_INST_WAITING = 1,   /* waiting_for_equil */
    MS_INST_EQUIL = 2,     /* transient: equilibrium reached this step */
    MS_INST_DONE = 3,      /* equilibrium reached at dial factor 1 */
    MS_INST_FAILED = 4     /* force guard tripped */
};

typedef struct ms_batch_instance {
    ms_mesh_desc mesh;
    ms_params params;
    /* Protocol-3 programmed field, T x 3 row-major (director angle,
     * lambda_final, nu_ot), as abar_info of do_dialling.cpp:112-123;
     * lambda_final and nu_ot must be the same on every triangle. */
    const double* abar_info;
    double timestep;
    double damping_factor_1, damping_factor_2;  /* dialling, waiting */
    int64_t timesteps_per_dial_phase;
    int64_t timesteps_between_equil_checks;
    double dial_factors_to_hold_at_spacing;
    double dial_factor_to_start_from;
    int32_t stop_at_final_equilibrium;
    const double* dofs;        /* 3N initial positions, SoA */
    const double* velocities;  /* 3N or NULL (zero) */
} ms_batch_instance;

typedef struct ms_batch_inst_status {
    int32_t status;            /* ms_inst_status */
    int32_t equilibria;        /* equilibria reached so far */
    int64_t stepcount;
    double dial_factor, last_equil_dial, sim_time;
    double max_force_ratio, max_speed_ratio;  /* at the last check */
    int64_t max_force_node, max_speed_node;
    int64_t offending_dof;     /* failed: dof (SoA, within the instance) whose force tripped the guard, else -1 */
} ms_batch_inst_status;

/* Launch schedule: threads per block of the per-triangle kernel (0: the
 * persistent kernel fed by bulk-copied 128-triangle tiles; -1: the
 * node-tiled one-kernel step, node_block ignored -- the default when the
 * union has a node tile for every resident block, else 0) and of the
 * per-node kernel, steps per captured graph (even).  nodes_per_tile and
 * blocks_per_sm describe the node-tiled plan in use (read by
 * ms_batch_get_schedule, chosen by ms_batch_autotune; ignored by
 * ms_batch_set_schedule). */
typedef struct ms_batch_schedule {
    int32_t tri_block, node_block, chunk_steps;
    int32_t nodes_per_tile, blocks_per_sm;
} ms_batch_schedule;

/* Only dialling protocol 3 without ansatz dialling and Newtonian dynamics
 * (no gradient-descent steps) are batched. */
ms_status ms_batch_create(const ms_batch_instance* instances, int32_t n_instances, int32_t device,
                          int32_t precision, ms_batch** out);
void ms_batch_destroy(ms_batch* b);
const char* ms_batch_last_error(const ms_batch* b);
/* Runs up to max_steps steps, or until every instance is done or failed;
 * *steps_done receives the steps run. */
ms_status ms_batch_run(ms_batch* b, int64_t max_steps, int64_t* steps_done);
ms_status ms_batch_status(ms_batch* b, int32_t instance, ms_batch_inst_status* out);
/* Current (or final) positions and velocities of one instance, SoA; either may be NULL. */
ms_status ms_batch_download_dofs(ms_batch* b, int32_t instance, double* dofs, double* velocities);
/* Replaces one instance's positions (and velocities; NULL = zero), e.g. a
 * warm start, and restarts its state machine from dial_factor_to_start_from. */
ms_status ms_batch_upload_dofs(ms_batch* b, int32_t instance, const double* dofs, const double* velocities);
/* Restarts one instance's state machine at dial_factor: dialling from there
 * (waiting = 0, as dial_factor_to_start_from), or waiting for equilibrium
 * with the programmed metric held at dial_factor (waiting = 1; for a warm
 * start uploaded with ms_batch_upload_dofs, which itself restarts from
 * dial_factor_to_start_from, so call this after it). */
ms_status ms_batch_set_start(ms_batch* b, int32_t instance, double dial_factor, int32_t waiting);
ms_status ms_batch_set_schedule(ms_batch* b, const ms_batch_schedule* s);
ms_status ms_batch_get_schedule(const ms_batch* b, ms_batch_schedule* s);
/* Times every built-in schedule on this batch (steps_per_trial steps each,
 * CUDA events) from the current state, puts the state back after each trial,
 * and keeps the fastest; then rebuilds the node-tiled plan at other tile
 * sizes and resident blocks per SM, times each the same way and keeps the
 * fastest plan.  All schedules and plans give the same bits. */
ms_status ms_batch_autotune(ms_batch* b, int32_t steps_per_trial, ms_batch_schedule* chosen,
                            double* best_ms_per_step);
/* The last ms_batch_autotune's trials as text, one per line (schedule or
 * node-tiled plan, ms per step): copies up to len - 1 bytes and a NUL into
 * buf, returns the full length (-1 for a null batch). */
int32_t ms_batch_autotune_report(const ms_batch* b, char* buf, int32_t len);
ms_status ms_batch_info(const ms_batch* b, int64_t* num_nodes, int64_t* num_tris, int32_t* n_instances);
void* ms_batch_stream(ms_batch* b);

/* ---- coordinate network of the learned warm start ---------------------------
 * No reference counterpart: it replaces move_nodes_to_ansatz_positions
 * (main.cpp:226-230) as the source of an ansatz.  A SiLU MLP
 * in_dim -> width (x hidden_layers) -> out_dim; every layer runs on the
 * tensor cores (tcgen05, BF16 operands, FP32 accumulation); FP32 master
 * weights, Adam (beta 0.9 / 0.999, eps 1e-8), mean-squared-error loss.
 * Parameter layout (ms_mlp_get_params): per layer W [N][K] row-major, then
 * b [Np]; K is in_dim rounded up to 16 for the first layer (the extra
 * columns stay zero) and width after; N = width, or out_dim for the last
 * layer whose bias is padded to Np = 16. */
typedef struct ms_mlp ms_mlp;

ms_status ms_mlp_create(int32_t in_dim, int32_t width, int32_t hidden_layers, int32_t out_dim, uint64_t seed,
                        int32_t device, ms_mlp** out);
void ms_mlp_destroy(ms_mlp* h);
const char* ms_mlp_last_error(const ms_mlp* h);
ms_status ms_mlp_num_params(const ms_mlp* h, int64_t* n);
ms_status ms_mlp_get_params(ms_mlp* h, float* params);
ms_status ms_mlp_set_params(ms_mlp* h, const float* params);
/* y (n x out_dim) = network(x (n x in_dim)), host arrays, row-major. */
ms_status ms_mlp_forward(ms_mlp* h, const float* x, int64_t n, float* y);
/* Mean-squared-error loss of one batch (n <= 65536) and its gradient with
 * respect to every parameter (ms_mlp_get_params layout); no update. */
ms_status ms_mlp_loss_grad(ms_mlp* h, const float* x, const float* t, int64_t n, double* loss, float* grads);
/* Training set (n rows of in_dim inputs and out_dim targets) to the device. */
ms_status ms_mlp_set_data(ms_mlp* h, const float* x, const float* t, int64_t n);
/* epochs passes over the training set in shuffled batches of `batch` rows;
 * epoch_loss (epochs entries, may be NULL) gets each epoch's mean loss. */
ms_status ms_mlp_train(ms_mlp* h, int32_t epochs, int32_t batch, double lr, uint64_t seed, float* epoch_loss);
void* ms_mlp_stream(ms_mlp* h);

#ifdef __cplusplus
}

#include <stdexcept>

/* C++ callers: the reference's error convention (a std::runtime_error that
 * main.cpp catches, logs and turns into return -1; main.cpp:448-474).  A guard
 * trip carries the reference's own message, "implausibly_high_force"
 * (advance_dynamics.cpp:71); any other failure the handle's last error, or the
 * status name when there is no handle or no message. */
inline void ms_check(int rc, const ms_handle* h) {
    if (rc == MS_OK) return;
    if (rc == MS_ERR_IMPLAUSIBLE_FORCE) throw std::runtime_error("implausibly_high_force");
    const char* m = h ? ms_last_error(h) : nullptr;
    throw std::runtime_error(m && *m ? m : ms_status_string(rc));
}
#endif

#endif /* MORPHOSHELL_GPU_H */
