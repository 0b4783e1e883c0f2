// Device-side data layout and kernel entry points of the force-and-dynamics
// loop.  Shared by the kernels (kernels.cu) and the C ABI (capi.cu).
//
// Layout in HBM (N nodes, T triangles, all structure-of-arrays so that a warp
// reading one field of 32 consecutive triangles or nodes touches 256
// contiguous bytes):
//   pos[2][3][N], vel[2][3][N]   double, ping-pong state (step i reads buffer
//                                i&1, writes the other)
//   mass[N], fixed[N]            dof mass, constrained flag
//   patch[6][T]                  int32 patch node ids (3 vertices, 3 extra)
//   coef[24][T]                  derivative weights (see ms_mesh_desc)
//   area[T], thick[T], shear[T]  reference area, thickness, shear modulus
//   abar[3][T], bbar[3][T]       programmed tensors currently in force
//   info_a[ka][T], info_b[kb][T] CELL_DATA programmed fields (dialling input)
//   a0[3][T], b0[3][T]           a, b at zero dial factor
//   contrib[T][6][3]             per-(triangle, patch slot) force contribution
//   inc_off[N+1], inc_ent[6T]    for each node, the (6t+slot) entries that
//                                touch it, in ascending t (deterministic gather)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace msb {

constexpr int kMaxDialCols = 16;

// Error record written by kernels; a non-zero flag makes every later kernel
// of a multi-step launch return immediately.
struct DevError {
    int flag;                       // 0 ok, else an ms_status code
    int base;                       // global index of step 0 of the running graph chunk
    unsigned long long guard_key;   // (global step << 32) | dof of the first guard trip
};

// Result slot of the equilibrium reduction (is_at_equilibrium.cpp:62-84).
struct DevEquil {
    double max_force;
    double max_speed;
    long long max_force_node;
    long long max_speed_node;
};

// Per-block partial of the equilibrium reduction.
struct EqPartial {
    double f;
    double v;
    int fn;
    int vn;
};

// Everything a kernel may need, passed by value.
struct DevMesh {
    int N, T;
    const int* patch;
    const double* coef;
    const double* area;
    const double* thick;
    const double* shear;
    const double* mass;
    const unsigned char* fixed;
    const unsigned char* boundary;
    const int* inc_off;
    const int* inc_ent;
    // programmed tensors
    double* abar;
    double* bbar;
    const double* info_a;
    const double* info_b;
    int ka, kb;
    const double* a0;
    const double* b0;
    // uniform material (used when uniform_hmu)
    int uniform_hmu;
    double h_uniform, mu_uniform;
    // constants
    double nu, gamma;
    // float copies for the mixed-precision path (may be null)
    const float* coef_f;
    const float* area_f;
    float* contrib_f;
};

struct DevState {
    double* pos[2];
    double* vel[2];
    double* forces;   // [3][N], used by the one-call-per-function path
    double* cq;       // [T][15]
    double* dEdcq;    // [T][15]
    double* contrib;  // [T][18]
    DevError* err;
    DevEquil* equil;
    EqPartial* eq_part;
    unsigned int* eq_counter;
    int eq_blocks;
    const double* dials;  // per-step dial factors of the current launch
};

// Per-step scalars (baked into each captured kernel node).
struct StepScalars {
    int step;          // index within the graph chunk; + DevError::base = global step
    int parity;        // buffer read this step
    double dt;
    double damping;    // damping_factor
    double rho_hh;     // ref_density * min_ref_thickness * min_ref_thickness
    double force_limit;  // 50000 * char_force_scale
    int gd;            // gradient-descent dynamics
    int check;         // do the equilibrium reduction this step
};

enum DialMode { DIAL_ARRAYS = 0, DIAL_LCE = 3 };

// ---- launchers (kernels.cu) ------------------------------------------------
cudaError_t launch_tri_fused(const DevMesh& m, const DevState& s, const StepScalars& sc, int dial_mode,
                             int mixed, cudaStream_t st);
cudaError_t launch_node_update(const DevMesh& m, const DevState& s, const StepScalars& sc, int mixed,
                               cudaStream_t st);
cudaError_t launch_surface_derivs(const DevMesh& m, const DevState& s, int parity, cudaStream_t st);
cudaError_t launch_forces_from_cq(const DevMesh& m, const DevState& s, int write_dE, cudaStream_t st);
cudaError_t launch_gather_forces(const DevMesh& m, const DevState& s, cudaStream_t st);
cudaError_t launch_damping(const DevMesh& m, const DevState& s, int parity, double damping, double rho_hh,
                           cudaStream_t st);
cudaError_t launch_constraints(const DevMesh& m, const DevState& s, cudaStream_t st);
cudaError_t launch_equilibrium(const DevMesh& m, const DevState& s, int parity, cudaStream_t st);
cudaError_t launch_guard(const DevMesh& m, const DevState& s, double force_limit, cudaStream_t st);
cudaError_t launch_advance(const DevMesh& m, const DevState& s, int parity, double dt, double damping,
                           double rho_hh, int gd, cudaStream_t st);
cudaError_t launch_dialling(const DevMesh& m, int protocol, double dial, double spacing, int from_ansatz,
                            cudaStream_t st);
cudaError_t launch_a_b_normals(const DevMesh& m, const DevState& s, double* a, double* b, double* n,
                               cudaStream_t st);
// Output diagnostics from the current cq (surface derivs must be current).
cudaError_t launch_output_tri(const DevMesh& m, const DevState& s, double* curv, double* edens, double* strain,
                              double* stress, double* tri_energy /*[2][T]*/, cudaStream_t st);
cudaError_t launch_angle_deficits(const DevMesh& m, const DevState& s, int parity, double* out, cudaStream_t st);
cudaError_t launch_kinetic(const DevMesh& m, const DevState& s, int parity, double* ke /*[N]*/, cudaStream_t st);
// Advances DevError::base by `len` after a graph chunk of `len` steps.
cudaError_t launch_chunk_end(const DevState& s, int len, cudaStream_t st);
// Deterministic compensated sum of n doubles into *out (two passes, fixed order).
cudaError_t launch_comp_sum(const double* x, int n, double* partial /*>= 1024*/, double* out, cudaStream_t st);

}  // namespace msb
