// Node-tiled step (ms_set_step_path 3): the whole fused step in one kernel,
// with no per-triangle contributions in HBM.
//
// A persistent block walks node tiles (blockIdx.x, then every gridDim.x-th).
// For each tile it streams the chunk records of the tile's triangle list
// (every triangle whose patch touches one of the tile's nodes, ascending t).
// Thread 0 copies a record with two cp.async.bulk (the tables into the
// block's single table area, the node section into one of two slots;
// completion counted in bytes on one mbarrier).  The copy of the next record
// starts as soon as every thread holds its triangle's tables in registers,
// so it lands while the block computes: each thread forms one triangle's 18
// contributions (the arithmetic of the bulk-copy per-triangle kernel,
// tile_tri) and stages them in a field-major area, and then the chunk's runs
// add them to the tile's per-node accumulators in shared memory: one thread
// per run, a run being one node's entries in this chunk in ascending
// triangle order.  Chunks are taken in order, so each node's force is summed
// in ascending triangle order from zero -- the order, and so the bits, of
// the node kernel's gather (calc_deformation_forces.cpp:185).  After the
// tile's last chunk the block finishes its nodes (damping, constraints,
// guard, equilibrium maxima, symplectic Euler; node_core) and moves on.
//
// Cost against the two-kernel step: triangles on tile borders are computed
// once per tile they touch (about 20 % more triangle work at 700-node
// tiles), but the contribution round trip through HBM (144 B per triangle in
// FP64, 72 B mixed) and the node kernel's incidence lists disappear.
#include <algorithm>
#include <climits>

#include "internal.cuh"
#include "step_common.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tridev;
using namespace tiles;

// Nodes finished per thread with their loads in flight together (two spill
// at the register budget of 3 blocks per SM and were measured slower).
constexpr int kFinishBatch = 1;

// Shared memory of a block: the chunk's fixed part (ids, weights,
// trigonometry; single-buffered: it is refilled as soon as every thread holds
// its triangle's tables in registers), the contribution staging area, two
// node sections (the current chunk's, and the next one landing) and the
// tile's per-node accumulators.
template <bool MIXED>
struct NtSmem {
    static constexpr size_t fixed = TileLayout<MIXED>::bytes;
    static constexpr size_t stage = (size_t)kTile * 18 * (MIXED ? 4 : 8);
    __host__ __device__ static size_t ns_cap(size_t stride) { return stride - fixed; }
    __host__ __device__ static size_t bytes(size_t stride, int nodes) {
        return fixed + stage + 2 * ns_cap(stride) + 24 * (size_t)nodes;
    }
};

// Resident blocks asked of the compiler (registers): FP64 at 3 per SM (168
// registers), mixed at 4 (128).
#ifndef MSB_NT_MINB
#define MSB_NT_MINB 3
#endif
#ifndef MSB_NT_MINB_MIXED
#define MSB_NT_MINB_MIXED 4
#endif

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kTile, MIXED ? MSB_NT_MINB_MIXED : MSB_NT_MINB)
    k_node_tiles(const DevMesh m, const ClusterPlan p, const NodeTilePlan q, const DevState s, const StepScalars sc) {
    using R = typename Real<MIXED>::T;
    using L = TileLayout<MIXED>;
    using SM = NtSmem<MIXED>;
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid
    double dial = 0.0, lam = 0.0, pw = 0.0;
    if (DIAL == DIAL_LCE) {
        dial = s.dials[3 * gstep];
        lam = s.dials[3 * gstep + 1];
        pw = s.dials[3 * gstep + 2];
    }
    const double* pos = pos_buf(s, sc.parity);
    extern __shared__ __align__(128) unsigned char nt_smem[];
    __shared__ uint64_t bar;
    const size_t ns_cap = SM::ns_cap(q.stride);
    unsigned char* fx = nt_smem;
    R* stage = reinterpret_cast<R*>(nt_smem + SM::fixed);
    unsigned char* nsec = nt_smem + SM::fixed + SM::stage;
    double* acc = reinterpret_cast<double*>(nsec + 2 * ns_cap);
    const int i = threadIdx.x;
    for (int j = i; j < 3 * q.nodes; j += kTile) acc[j] = 0.0;
    if (i == 0) {
        bar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // Thread 0: chunk c's fixed part into the fixed area and its node section
    // into node-section slot `slot`, both counted on the one barrier.
    auto fetch = [&](int c, int slot) {
        const unsigned char* src = q.rec + (size_t)c * q.stride;
        const uint32_t nb = __ldg(q.chunk_bytes + c) - (uint32_t)SM::fixed;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)),
                     "r"((uint32_t)SM::fixed + nb)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(fx)),
                     "l"(src), "r"((uint32_t)SM::fixed), "r"(smem_addr(&bar))
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(nsec + slot * ns_cap)),
                     "l"(src + SM::fixed), "r"(nb), "r"(smem_addr(&bar))
                     : "memory");
    };
    // The triangle id of a slot is needed only for per-triangle material,
    // per-triangle LCE fields or programmed tensors read from arrays.
    const bool need_t = DIAL != DIAL_LCE || !p.lce_uniform || !m.uniform_hmu;
    double fmax = -1.0, vmax = -1.0;
    int fnode = INT_MAX, vnode = INT_MAX;
    int tile = blockIdx.x;  // the grid is at most the tile count
    int c = __ldg(q.tile_chunk + tile);
    if (i == 0) fetch(c, 0);
    uint32_t phase = 0u;
    int slot = 0;  // node-section slot of the current chunk
    bool failed = false;
    for (;;) {
        const int cend = __ldg(q.tile_chunk + tile + 1);
        const int ntile = tile + gridDim.x;
        const int cn = ntile < q.ntiles ? __ldg(q.tile_chunk + ntile) : -1;
        const int n0 = tile * q.nodes;
        const int nn = min(q.nodes, m.N - n0);
        for (; c < cend; ++c) {
            const int nc = c + 1 < cend ? c + 1 : cn;
            // This barrier also ends the previous chunk's runs, so the
            // staging area and the other node-section slot are free after it.
            const int ok = __syncthreads_and(bar_wait(&bar, phase) ? 1 : 0);
            phase ^= 1u;
            if (!ok) {
                // No other copy is in flight (the next one starts below).
                if (i == 0) atomicCAS(&s.err->flag, 0, 5);  // MS_ERR_TIMEOUT
                failed = true;
                break;
            }
            const unsigned char* ns = nsec + slot * ns_cap;
            const int4 hd = *reinterpret_cast<const int4*>(ns);  // R, E, ntri
            const int* sid = reinterpret_cast<const int*>(fx);
            const R* scoef = reinterpret_cast<const R*>(fx + L::ids);
            const double* saux = reinterpret_cast<const double*>(fx + L::ids + L::coef);
            int ids[6];
            R cf[24];
#pragma unroll
            for (int k = 0; k < 6; ++k) ids[k] = sid[k * kTile + i];
#pragma unroll
            for (int k = 0; k < 24; ++k) cf[k] = scoef[k * kTile + i];
            const double area = saux[i], c2 = saux[kTile + i], s2 = saux[2 * kTile + i], cs = saux[3 * kTile + i];
            const bool live = i < hd.z;
            const int t = (need_t && live) ? __ldg(q.chunk_tri + (size_t)c * kTile + i) : 0;
            // The table loads above may still be in flight (their values are
            // used after the barrier): order them before the bulk copy that
            // refills the area.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (i == 0 && nc >= 0) fetch(nc, slot ^ 1);
            R f[18];
#pragma unroll
            for (int j = 0; j < 18; ++j) f[j] = R(0);
            if (live) tile_tri<DIAL, MIXED>(m, p, pos, dial, lam, pw, t, ids, cf, area, c2, s2, cs, f);
#pragma unroll
            for (int k = 0; k < 18; ++k) stage[k * kTile + i] = f[k];
            __syncthreads();
            // Runs: one node's entries of this chunk each, distinct nodes, so
            // the runs of a chunk add in parallel without conflicts.
            {
                // Staging is field-major: component k of patch slot sl of
                // the chunk's triangle i at stage[(3 sl + k) kTile + i]; an
                // entry holds sl * 3 kTile + i.
                const unsigned short* rn = reinterpret_cast<const unsigned short*>(ns + 16);
                const unsigned short* re = rn + hd.x;
                const unsigned short* en = re + hd.x;
                for (int r = i; r < hd.x; r += kTile) {
                    const int j = rn[r];
                    int e = r ? re[r - 1] : 0;
                    const int e1 = re[r];
                    double a0 = acc[3 * j], a1 = acc[3 * j + 1], a2 = acc[3 * j + 2];
                    for (; e < e1; ++e) {
                        const R* v = stage + en[e];
                        a0 += (double)v[0];
                        a1 += (double)v[kTile];
                        a2 += (double)v[2 * kTile];
                    }
                    acc[3 * j] = a0;
                    acc[3 * j + 1] = a1;
                    acc[3 * j + 2] = a2;
                }
            }
            slot ^= 1;
        }
        if (failed) break;
        // The tile's nodes: every contribution is in once the runs of the
        // last chunk are done.  Each thread clears the accumulators it reads,
        // ready for the next tile (whose first runs come after at least two
        // more block barriers).
        __syncthreads();
        for (int j0 = 0; j0 < nn; j0 += kTile * kFinishBatch) {
            NodeIn in[kFinishBatch];
#pragma unroll
            for (int b = 0; b < kFinishBatch; ++b) {
                const int j = j0 + b * kTile + i;
                if (j < nn) in[b] = node_load(m, s, sc, n0 + j);
            }
#pragma unroll
            for (int b = 0; b < kFinishBatch; ++b) {
                const int j = j0 + b * kTile + i;
                if (j < nn) {
                    const double Fx = acc[3 * j], Fy = acc[3 * j + 1], Fz = acc[3 * j + 2];
                    acc[3 * j] = acc[3 * j + 1] = acc[3 * j + 2] = 0.0;
                    node_core(m, s, sc, gstep, n0 + j, in[b], Fx, Fy, Fz, fmax, fnode, vmax, vnode);
                }
            }
        }
        tile = ntile;
        if (tile >= q.ntiles) break;
        c = cn;
    }
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
