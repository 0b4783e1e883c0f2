// Per-triangle kernel of the two-kernel step fed by bulk asynchronous
// copies (ms_set_step_path 2).
//
// The per-triangle tables are regrouped into tiles of kTile triangles, each
// tile one contiguous record: patch ids [6][kTile] int32, derivative weights
// [24][kTile] (double, or float for the mixed path), director trigonometry
// and area [4][kTile] double (area, cos^2, sin^2, cos sin).  A persistent
// block walks its tiles; thread 0 copies the next tile's record into the
// other half of a double buffer with one cp.async.bulk (completion counted
// in bytes on an mbarrier) while the block computes the current one, so the
// ~250 B of tables per triangle stream in while the node positions are
// gathered and the forces computed.  Inside a tile, field k of triangle i
// sits at [k][i], so the per-thread shared-memory reads are conflict free.
// Contributions leave through the consumed weight area as contiguous runs.
#include <algorithm>

#include "internal.cuh"
#include "step_common.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tridev;
using namespace tiles;

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kTile) k_tri_tiles(const DevMesh m, const ClusterPlan p, const DevState s,
                                                   const StepScalars sc) {
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
    const unsigned char* tl = reinterpret_cast<const unsigned char*>(MIXED ? p.tiles_f : p.tiles);
    R* out;
    if constexpr (MIXED) out = m.contrib_f;
    else out = s.contrib;
    tile_loop<MIXED>(m.T, tl, out, &s.err->flag,
                     [&](int t, const int (&ids)[6], const R (&c)[24], double area, double c2, double s2, double cs,
                         R (&f)[18]) { tile_tri<DIAL, MIXED>(m, p, pos, dial, lam, pw, t, ids, c, area, c2, s2, cs, f); });
}

template <int DIAL, bool MIXED>
cudaError_t launch_one(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                       cudaStream_t st) {
    constexpr int smem = 2 * TileLayout<MIXED>::bytes;
    const int ntiles = (m.T + kTile - 1) / kTile;
    const int grid = std::min(ntiles, p.tile_grid);
    if (grid <= 0) return cudaSuccess;
    k_tri_tiles<DIAL, MIXED><<<grid, kTile, smem, st>>>(m, p, s, sc);
    return cudaGetLastError();
}

template <int DIAL, bool MIXED>
cudaError_t prepare_one(int& blocks) {
    constexpr int smem = 2 * TileLayout<MIXED>::bytes;
    cudaError_t e = cudaFuncSetAttribute(k_tri_tiles<DIAL, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_tri_tiles<DIAL, MIXED>, kTile, smem);
    if (e != cudaSuccess) return e;
    blocks = blocks == 0 ? b : std::min(blocks, b);
    return cudaSuccess;
}

}  // namespace

size_t tile_record_bytes(int mixed) { return mixed ? TileLayout<true>::bytes : TileLayout<false>::bytes; }

cudaError_t prepare_tile_kernels(int mixed, int* blocks_per_sm) {
    int b = 0;
    cudaError_t e = mixed ? prepare_one<DIAL_LCE, true>(b) : prepare_one<DIAL_LCE, false>(b);
    if (e == cudaSuccess) e = mixed ? prepare_one<DIAL_ARRAYS, true>(b) : prepare_one<DIAL_ARRAYS, false>(b);
    *blocks_per_sm = b;
    return e;
}

cudaError_t launch_tri_tiles(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                             int dial_mode, int mixed, cudaStream_t st) {
    if (dial_mode == DIAL_LCE)
        return mixed ? launch_one<DIAL_LCE, true>(m, p, s, sc, st) : launch_one<DIAL_LCE, false>(m, p, s, sc, st);
    return mixed ? launch_one<DIAL_ARRAYS, true>(m, p, s, sc, st) : launch_one<DIAL_ARRAYS, false>(m, p, s, sc, st);
}

}  // namespace msb
