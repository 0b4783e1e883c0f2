// Node-tiled step (ms_set_step_path 3): the whole fused step in one kernel,
// with no per-triangle contributions in HBM.
//
// A persistent block walks node tiles (blockIdx.x, then every gridDim.x-th).
// For each tile it walks the chunk records of the tile's triangle list
// (every triangle whose patch touches one of the tile's nodes, ascending t).
// Each thread reads its slot's tables (ids, weights, trigonometry) straight
// into registers -- the next chunk's while the block adds up the current
// one's runs -- and thread 0 bulk-copies the chunk's node section into one
// of two shared-memory slots (completion counted in bytes on one mbarrier).
// Each thread forms one triangle's 18 contributions (the arithmetic of the
// bulk-copy per-triangle kernel, tile_tri) and stages them in a field-major
// area, and then the chunk's runs add them to the tile's per-node
// accumulators in shared memory: one thread per run, a run being one node's
// entries in this chunk in ascending triangle order.  Chunks are taken in
// order, so each node's force is summed in ascending triangle order from
// zero -- the order, and so the bits, of the node kernel's gather
// (calc_deformation_forces.cpp:185).  After the tile's last chunk the block
// finishes its nodes (damping, constraints, guard, equilibrium maxima,
// symplectic Euler; node_core) and moves on.
//
// Cost against the two-kernel step: triangles on tile borders are computed
// once per tile they touch (about 20 % more triangle work at 700-node
// tiles), but the contribution round trip through HBM (144 B per triangle in
// FP64, 72 B mixed) and the node kernel's incidence lists disappear.
#include <algorithm>
#include <climits>

#include "internal.cuh"
#include "step_common.cuh"
#include "node_tile_walk.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tridev;
using namespace tiles;

// Resident blocks asked of the compiler (registers): FP64 at 3 per SM (168
// registers; at 4 it spills and was measured slower), mixed at 5 (96, no
// spills; 2.4 % faster than 4, while 6 spills and is slower).
#ifndef MSB_NT_MINB
#define MSB_NT_MINB 3
#endif
#ifndef MSB_NT_MINB_MIXED
#define MSB_NT_MINB_MIXED 5
#endif

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kTile, MIXED ? MSB_NT_MINB_MIXED : MSB_NT_MINB)
    k_node_tiles(const DevMesh m, const ClusterPlan p, const NodeTilePlan q, const DevState s, const StepScalars sc) {
    using R = typename Real<MIXED>::T;
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid
    double dial = 0.0, lam = 0.0, pw = 0.0;
    if (DIAL == DIAL_LCE) {
        dial = s.dials[3 * gstep];
        lam = s.dials[3 * gstep + 1];
        pw = s.dials[3 * gstep + 2];
    }
    const double* pos = pos_buf(s, sc.parity);
    // The triangle id of a slot is needed only for per-triangle material,
    // per-triangle LCE fields or programmed tensors read from arrays.
    const bool need_t = DIAL != DIAL_LCE || !p.lce_uniform || !m.uniform_hmu;
    double fmax = -1.0, vmax = -1.0;
    int fnode = INT_MAX, vnode = INT_MAX;
    node_tile_walk<MIXED>(
        q, m.N, need_t, &s.err->flag,
        [&](int t, int, const int (&ids)[6], const R (&cf)[24], double area, double c2, double s2, double cs,
            R (&f)[18]) {
            tile_tri<DIAL, MIXED>(m, p, pos, dial, lam, pw, t, ids, cf, area, c2, s2, cs, f);
        },
        [&](int n, double Fx, double Fy, double Fz) {
            node_core(m, s, sc, gstep, n, node_load(m, s, sc, n), Fx, Fy, Fz, fmax, fnode, vmax, vnode);
        });
    if (sc.check) {
        const EqPartial r = eq_block_reduce<kTile>(fmax, fnode, vmax, vnode);
        eq_store_and_fold(s, r, blockIdx.x, gridDim.x, gridDim.x);
    }
}

template <int DIAL, bool MIXED>
cudaError_t launch_one(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                       const StepScalars& sc, cudaStream_t st) {
    const int grid = std::min(q.ntiles, q.grid);
    if (grid <= 0) return cudaSuccess;
    k_node_tiles<DIAL, MIXED><<<grid, kTile, NtSmem<MIXED>::bytes(q.stride, q.nodes), st>>>(m, p, q, s, sc);
    return cudaGetLastError();
}

template <int DIAL, bool MIXED>
cudaError_t prepare_one(size_t smem, int& blocks) {
    cudaError_t e =
        cudaFuncSetAttribute(k_node_tiles<DIAL, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_node_tiles<DIAL, MIXED>, kTile, smem);
    if (e != cudaSuccess) return e;
    blocks = blocks == 0 ? b : std::min(blocks, b);
    return cudaSuccess;
}

}  // namespace

size_t node_tile_smem(size_t stride, int nodes, int mixed) {
    return mixed ? NtSmem<true>::bytes(stride, nodes) : NtSmem<false>::bytes(stride, nodes);
}

int node_tile_blocks_target(int mixed) { return mixed ? MSB_NT_MINB_MIXED : MSB_NT_MINB; }

cudaError_t prepare_node_tile_kernels(int mixed, size_t smem, int* blocks_per_sm) {
    int b = 0;
    cudaError_t e = mixed ? prepare_one<DIAL_LCE, true>(smem, b) : prepare_one<DIAL_LCE, false>(smem, b);
    if (e == cudaSuccess) e = mixed ? prepare_one<DIAL_ARRAYS, true>(smem, b) : prepare_one<DIAL_ARRAYS, false>(smem, b);
    *blocks_per_sm = b;
    return e;
}

cudaError_t launch_node_tiles(const DevMesh& m, const ClusterPlan& p, const NodeTilePlan& q, const DevState& s,
                              const StepScalars& sc, int dial_mode, int mixed, cudaStream_t st) {
    if (dial_mode == DIAL_LCE)
        return mixed ? launch_one<DIAL_LCE, true>(m, p, q, s, sc, st) : launch_one<DIAL_LCE, false>(m, p, q, s, sc, st);
    return mixed ? launch_one<DIAL_ARRAYS, true>(m, p, q, s, sc, st) : launch_one<DIAL_ARRAYS, false>(m, p, q, s, sc, st);
}

}  // namespace msb
