/*
 * oracle.h -- C ABI shared by the two CPU oracles (TEST INFRASTRUCTURE ONLY).
 *
 *   orc_*  libmorpho_oracle.so : this project's C++ restatement of the
 *          reference's per-step algorithm (morpho_oracle.cpp)
 *   ref_*  _ref/libmorpho_ref.so : the reference's own source files,
 *          compiled unmodified against eigen_shim/, driven by ref_bridge.cpp
 *
 * Only tests, the smoke check and the CPU-baseline leg of the benchmark use
 * these; the product never links them.  Arrays: positions N x 3 row-major,
 * patch T x 6 (3 vertices then 3 extra patch nodes), mat2 T x 18 (the 6 x 3
 * patch matrix, row-major), coeffs T x 24 (ms_mesh_desc layout), dofs /
 * velocities / forces SoA [X(N)|Y(N)|Z(N)], cq and dE 15 per triangle.
 * scal[9] = {nu, gamma, ref_density, min_ref_thickness, char_force_scale,
 *            char_speed_scale, force_threshold, speed_threshold, unused}.
 */
#ifndef MORPHO_ORACLE_H
#define MORPHO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_API(P)                                                                                            \
    void* P##_create(int N, int T, const double* ref_pos, const int32_t* patch, const double* mat2,             \
                     const double* coeffs, const double* mass, const double* area, const double* thick,         \
                     const double* shear, const uint8_t* fixed, const uint8_t* boundary, const double* scal);     \
    void P##_destroy(void* c);                                                                                   \
    int P##_set_programmed(void* c, int protocol, const double* abar_info, int ka, const double* bbar_info,     \
                           int kb, double spacing, int from_ansatz);                                            \
    void P##_set_zero_dial_state(void* c, const double* a0, const double* b0);                                   \
    void P##_set_state(void* c, const double* dofs, const double* vel);                                          \
    void P##_get_state(void* c, double* dofs, double* vel);                                                      \
    void P##_get_forces(void* c, double* forces);                                                                \
    void P##_do_dialling(void* c, double dial);                                                                  \
    void P##_get_programmed(void* c, double* abar, double* bbar);                                                \
    void P##_surface_derivs(void* c, double* cq);                                                                \
    void P##_a_b_normals(void* c, double* a, double* b, double* n);                                              \
    void P##_deformation_forces(void* c, double* forces, double* dE);                                            \
    void P##_non_deformation_forces(void* c, double damping, int gd);                                            \
    void P##_impose_constraints(void* c);                                                                        \
    int P##_is_at_equilibrium(void* c, double* out4);                                                            \
    int P##_advance_dynamics(void* c, double dt, double damping, int gd, int64_t* bad_dof, double* bad_force);   \
    int P##_step_n(void* c, int n, const double* dials, double dt, double damping, int gd, int* steps_done);     \
    void P##_output_quantities(void* c, double* curv, double* edens, double* strains, double* stresses,          \
                               double* deficits, double* energies);                                              \
    void P##_set_threads(int n);

ORACLE_API(orc)
ORACLE_API(ref)

/* The reference's own set-up (main.cpp:91-209) from a settings file and a
 * mesh file; ref_* only. */
int ref_setup_from_files(const char* settings, const char* vtk, int* N_out, int* T_out, int32_t* patch,
                         double* mat2, double* masses, double* dofs0, double* scal, char* err, int len);
int ref_setup_full(const char* settings, const char* vtk, int* N_out, int* T_out, int32_t* patch, double* mat2,
                   double* masses, double* dofs0, double* scal, double* ref_pos, double* area, double* thick,
                   double* shear, uint8_t* fixed, uint8_t* boundary, char* err, int len);

#ifdef __cplusplus
}
#endif

#endif
