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
//   sell_off, sell_ent           the same lists in slices of 32 nodes, entry-
//                                major within a slice (coalesced index loads)
#pragma once

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

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
    // The same lists sliced for the node kernel (sliced ELL, 32 nodes a
    // slice): slice w holds nodes 32w .. 32w+31; its entries start at
    // sell_off[w], entry k of node 32w+lane is sell_ent[sell_off[w] + 32k +
    // lane] (ascending t, then -1 padding up to the slice's longest list).
    const int* sell_off;
    const int* sell_ent;
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
    double ks_uniform, kb_uniform, igmh_uniform;  // dev::material_coefs of the uniform material
    // constants
    double nu, gamma;
    // float contributions of the mixed-precision path (null otherwise)
    float* contrib_f;
};

// Cluster-tiled step (cluster.cu).  The triangles, in their Morton order, are
// cut into tiles of cs * tpc consecutive triangles, one tile per thread-block
// cluster of cs CTAs, tpc triangles per CTA.  A node whose every patch
// incidence lies in one tile is "owned" by that tile: its force is summed from
// the cluster's shared memory and it is updated by the same kernel.  Every
// other node is a "halo" node: the contributions it receives are written to
// HBM and a second kernel sums them.  Both sums run in ascending triangle
// order, the order of the two-kernel path.
struct ClusterPlan {
    int cs;                    // CTAs per cluster (1..8)
    int tpc;                   // triangles per CTA (<= 1024)
    int nclusters;
    int threads;               // threads per CTA
    const int4* tri_idx;       // [T][2] int4: 6 patch ids, halo-slot mask, unused
    const double* coef_aos;    // [T][24] derivative weights, per triangle contiguous
    const float* coef_aos_f;   // [T][24] float copy (mixed precision)
    const double4* tri_aux;    // [T]: area, cos^2, sin^2, cos*sin of the director angle
    const double2* lce_ln;     // [T]: lambda_final, nu_ot (only when not uniform)
    int lce_uniform;           // lambda_final and nu_ot equal on every triangle
    const int* own_base;       // [nclusters + 1] range of each tile's owned nodes in own_nodes
    const int* own_nodes;      // owned node ids, grouped by tile, ascending within a tile
    const int* own_off;        // [n_owned + 1] offsets into own_ent
    const unsigned short* own_ent;  // (rank << 13) | (index in CTA << 3) | slot, ascending triangle
    const int* halo_nodes;     // nodes summed by the halo kernel
    int n_halo;
    // Tile records of the bulk-copy-fed per-triangle kernel (tri_tiles.cu):
    // per kTile triangles, ids [6][kTile] int32, weights [24][kTile]
    // (double; float in tiles_f), area and director trigonometry
    // [4][kTile] double.
    const void* tiles;
    const void* tiles_f;
    int tile_grid;             // persistent blocks (SMs x resident blocks)
};

// Triangles per tile of the bulk-copy-fed per-triangle kernel.
constexpr int kTile = 128;
// Node-tiled step: the flag of a node's last run in its tile, and the
// largest tile the 15 remaining bits of a run's node index can address.
constexpr unsigned short kRunFinal = 0x8000;
constexpr int kNtMaxNodes = 32768;

// Node-tiled step (node_tiles.cu): one kernel per step.  The nodes, in their
// Morton order, are cut into node tiles of `nodes` consecutive nodes.  The
// triangles whose patch touches a node tile (every triangle that contributes
// to one of its nodes, in ascending triangle order) are that tile's list; a
// triangle near a tile border is on the lists of every tile it touches and is
// computed once for each.  A list is cut into chunks of kTile triangles, each
// one record: the tile record of the bulk-copy kernel (ids [6][kTile], weights
// [24][kTile], area and director trigonometry [4][kTile]) followed by the
// chunk's node section:
//   int32 header {R, E, ntri, 0}
//   uint16 run_node[R]   node (index in the tile) of each run; kRunFinal
//                        set on the node's last run in its tile (an empty
//                        one for a node with no triangles)
//   uint16 run_end[R]    end of the run's entries (exclusive, cumulative)
//   uint16 ent[E]        patch slot * 3 kTile + slot in chunk, per node ascending t
//                        (the x component of the contribution in the block's
//                        field-major staging area; y and z follow kTile apart)
//   uint16 slice_off[S]  the same entries in sliced order, for the
//                        warp-specialised step: runs 32s .. 32s + 31 form
//                        slice s (runs go longest first), and entry u of run
//                        r sits at slice_off[r / 32] + 32 u + r % 32
//   uint16 dst[6][kTile] for patch slot sl of the chunk's triangle i, the
//                        sliced position of its contribution (0xFFFF when
//                        the node is not in the tile)
// with the header {R, E, ntri, S}.  A block sums a node's contributions run
// by run, chunk by chunk, so every node's force is the sum in ascending
// triangle order, as in the node kernel.
struct NodeTilePlan {
    int nodes;                       // nodes per tile
    int ntiles;
    int nchunks;
    int grid;                        // persistent blocks of the node-tiled kernel (path 3)
    int grid_pipe;                   // persistent blocks of the warp-specialised kernel (path 4)
    size_t stride;                   // bytes between chunk records
    const unsigned char* rec;        // [nchunks] records (double weights, or float for mixed)
    const int* tile_chunk;           // [ntiles + 1] first chunk of each tile
    const unsigned* chunk_bytes;     // [nchunks] bytes to copy of each record (multiple of 16)
    const int* chunk_tri;            // [nchunks][kTile] triangle of each slot, -1 past the chunk's end
    const int* chunk_tag;            // [nchunks][kTile] the caller's value per slot (a batch: the instance), or null
    int slc;                         // entries of the sliced staging area (NodeTileLayout::slc_max)
};

// Host-side layout of a node-tile plan for tiles of NT consecutive nodes
// (node_tile_plan.cu): every tile's triangle list (ascending t), its chunks
// and their node sections, each chunk checked against the bounds the kernels
// rely on (entries inside the chunk's live slots, run nodes inside the tile,
// run ends ascending, everything inside one record).
struct NodeTileLayout {
    int K = 0, C = 0;
    std::vector<long long> start;   // [K + 1] list offsets into lst
    std::vector<int> lst;           // triangle lists, tile after tile
    std::vector<int> tile_chunk;    // [K + 1]
    std::vector<std::vector<unsigned short>> run_node, run_end, cent;  // per chunk
    std::vector<unsigned> bytes;    // [C] bytes to copy (fixed part + node section)
    size_t fixed = 0, stride = 0, ns_max = 0;
    std::vector<std::vector<unsigned short>> slice_off, dst;  // per chunk (sliced staging)
    int slc_max = 0;                // largest sliced staging of a chunk (entries, multiple of 32)
    bool sliced = false;            // records carry slice_off and dst (the warp-specialised step)
    size_t stride_sliced = 0;       // the record stride with them
};
// off/ent: each node's (6t + slot) entries in ascending order (CSR).
// sliced: the records carry the sliced order (slice_off, dst) that the
// warp-specialised step reads; the node-tiled step and the batch do not
// need it.
bool node_tile_layout(const int* patch_ids, int N, int T, int NT, int mixed, const std::vector<int>& off,
                      const std::vector<int>& ent, NodeTileLayout& L, std::string& err, int sliced = 0);
// A block walks its tiles in turn, so a step takes as long as the block with
// the most tiles: the tile size is chosen (between nt_min and nt_max nodes)
// so that the tile count is a multiple of sms x target blocks, at the largest
// size whose blocks still reach `target` per SM; blocks_for(shared bytes)
// sets up the kernel and returns its resident blocks per SM (0 when it
// cannot run).  On return `blocks` is the resident blocks of the chosen plan
// (0: the kernel cannot run); false with err for inconsistent lists.
// smem_for(layout, nodes) is the kernel's shared memory per block for a
// layout.
bool choose_node_tiles(const int* patch_ids, int N, int T, int mixed, int sms, int target, int nt_max, int nt_min,
                       const std::vector<int>& off, const std::vector<int>& ent,
                       const std::function<size_t(const NodeTileLayout&, int)>& smem_for,
                       const std::function<int(size_t)>& blocks_for, NodeTileLayout& L, int& NT, int& blocks,
                       std::string& err, int sliced = 0);
// The chunk records of a layout (ids from patch_ids [T][6]; weights from
// coef_d [T][24] double, or coef_f float for the mixed path when given; the
// trigonometry block from aux4 [T][4] = area, cos^2, sin^2, cos sin, or
// when null area with cos^2 = 1) and the triangle of every slot.
void fill_node_tile_records(const NodeTileLayout& L, const int* patch_ids, const double* coef_d, const float* coef_f,
                            const double* area, const double* aux4, int mixed, std::vector<unsigned char>& buf,
                            std::vector<int>& chunk_tri);
// Only the node sections (chunk c's at sections[pitch c], pitch at least
// the record's node-section room) and the triangle of every slot: the
// tables part of the records is then gathered on the device
// (batch.cu: fill_tables_on_device).
void fill_node_sections(const NodeTileLayout& L, size_t pitch, std::vector<unsigned char>& sections,
                        std::vector<int>& chunk_tri);

// Layout of the per-(triangle, slot) force contributions: x, y, z doubles;
// for the mixed path x, y, z floats, optionally padded with a zero to 16
// bytes so that the node kernel loads each with one vector load.
#ifndef MSB_MIXED_PAD4
#define MSB_MIXED_PAD4 0
#endif
constexpr int kMixedSlot = MSB_MIXED_PAD4 ? 4 : 3;
template <bool MIXED>
__host__ __device__ constexpr int contrib_slot() {
    return MIXED ? kMixedSlot : 3;
}
template <bool MIXED>
__host__ __device__ constexpr int contrib_stride() {
    return 6 * contrib_slot<MIXED>();
}

// ---- batched ensembles (batch.cu) ----------------------------------------------
// Many meshes stepped together: their tables are concatenated into one union
// mesh (nodes and triangles of instance i contiguous), every triangle and
// node carries its instance id, and each instance keeps its own parameters
// and its own copy of the main loop's state machine (main.cpp:269-508), run
// on the device so that long stretches need no host round trip.
struct InstParams {
    double dt, damping1, damping2, rho_hh, force_limit;
    double nu, gamma;
    double h, mu;                  // used when uniform_hmu
    double ks, kb, igmh;           // dev::material_coefs of (h, mu), used when uniform_hmu
    double char_force, char_speed, force_thresh, speed_thresh;
    double spacing;                // dial_factors_to_hold_at_spacing
    double lam_final, nu_ot;       // protocol-3 field (uniform per instance)
    long long steps_per_phase, steps_between_checks;
    int node_begin, node_end;      // union node range
    int uniform_hmu;
    int stop_at_final;
};

enum InstStatus { INST_DIALLING = 0, INST_WAITING = 1, INST_EQUIL = 2, INST_DONE = 3, INST_FAILED = 4 };

struct InstState {
    int status;
    int check_now;             // this step carries an equilibrium check
    int equilibria;
    int frozen_parity;         // buffer holding a done / failed instance's state, else -1
    long long k_phase, tsc, stepcount;
    double dial_factor, last_equil_dial, time, damping;
    double cur_dial, cur_lam, cur_pw;  // protocol-3 values of the last dialled step
    double max_force, max_speed;       // at the last check
    long long max_force_node, max_speed_node;
    unsigned long long guard_key;      // smallest tripping dof (within the instance) of this step, ~0 if none
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

// ---- cluster-tiled step (cluster.cu) ------------------------------------------
// dial_mode: DIAL_ARRAYS reads abar/bbar; DIAL_LCE evaluates protocol 3 from
// the per-step triple s.dials[3 * step] = {dial, lambda, lambda^(-2 nu)}.
cudaError_t launch_cluster_step(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                                int dial_mode, int mixed, cudaStream_t st);
cudaError_t launch_halo_update(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                               int mixed, cudaStream_t st);
// Two-kernel path, per-triangle kernel over the per-triangle (AoS) tables;
// with mixed, contributions go to DevMesh::contrib_f as float.
cudaError_t launch_tri_aos(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                           int dial_mode, int mixed, cudaStream_t st);
// Bulk-copy-fed per-triangle kernel (tri_tiles.cu): bytes of one tile
// record, kernel set-up (dynamic shared memory; resident blocks per SM) and
// launch.
size_t tile_record_bytes(int mixed);
cudaError_t prepare_tile_kernels(int mixed, int* blocks_per_sm);
cudaError_t launch_tri_tiles(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                             int dial_mode, int mixed, cudaStream_t st);
// Node-tiled step (node_tiles.cu): shared memory per block for a plan,
// kernel set-up (dynamic shared memory; resident blocks per SM) and launch.
size_t node_tile_smem(size_t stride, int nodes, int mixed);
// Warp-specialised node-tiled step (node_pipe.cu): shared memory per block,
// kernel set-up (resident blocks per SM), launch.
size_t node_pipe_smem(size_t stride, int nodes, int slc, int mixed);
cudaError_t prepare_node_pipe_kernels(int mixed, size_t smem, int* blocks_per_sm);
cudaError_t launch_node_pipe(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                             const StepScalars& sc, int dial_mode, int mixed, cudaStream_t st);
int node_tile_blocks_target(int mixed);
cudaError_t prepare_node_tile_kernels(int mixed, size_t smem, int* blocks_per_sm);
cudaError_t launch_node_tiles(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                              const StepScalars& sc, int dial_mode, int mixed, cudaStream_t st);
// Largest cluster size (8, 4, 2, 1) whose clusters fill the most SMs, and the
// CTA shape used with it.
int choose_cluster_size(int tpc, int threads, int mixed);
// Shared-memory bytes per CTA of the cluster kernel.
size_t cluster_smem_bytes(int tpc, int mixed);
// Threads per CTA of the cluster kernel.
int cluster_threads();
// Raise the dynamic shared-memory limit of the cluster kernels (once, outside
// any stream capture).
cudaError_t prepare_cluster_kernels(int tpc);
// Deterministic compensated sum of n doubles into *out (two passes, fixed order).
// Sliced-ELL copy of the incidence lists (see DevMesh::sell_off): offsets
// [ceil(N/32) + 1] and entries, built on the host from the CSR lists.
void build_sell(int N, const int* off, const int* ent, std::vector<int>& sell_off, std::vector<int>& sell_ent);
cudaError_t launch_comp_sum(const double* x, int n, double* partial /*>= 1024*/, double* out, cudaStream_t st);

}  // namespace msb
