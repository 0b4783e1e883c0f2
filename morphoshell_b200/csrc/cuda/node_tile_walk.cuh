// The chunk walk of the node-tiled step, shared by the single-mesh kernel
// (node_tiles.cu) and the batched one (batch.cu).  A block takes node tiles
// blockIdx.x, then every gridDim.x-th; for each tile it streams the chunk
// records of the tile's triangle list (NodeTilePlan), calls
//   tri(t, ids, c, area, c2, s2, cs, f)
// for every live triangle slot (t its triangle when need_t, else 0; f the 18
// contributions, zero on entry), adds the contributions to the tile's node
// accumulators run by run in ascending triangle order, and after the tile's
// last chunk calls
//   node(n, Fx, Fy, Fz)
// for each node of the tile with its summed deformation force.  A copy that
// does not land within the bounded wait sets *err_flag to 5 (MS_ERR_TIMEOUT)
// when it was 0 and ends the walk.
#pragma once

#include <cstdint>

#include "internal.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace tiles {

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

template <bool MIXED, typename Tri, typename Node>
__device__ __forceinline__ void node_tile_walk(const NodeTilePlan& q, int N, bool need_t, int* err_flag, Tri tri,
                                               Node node) {
    using R = typename tridev::Real<MIXED>::T;
    using L = TileLayout<MIXED>;
    using SM = NtSmem<MIXED>;
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
    int tile = blockIdx.x;  // the grid is at most the tile count
    int c = __ldg(q.tile_chunk + tile);
    if (i == 0) fetch(c, 0);
    uint32_t phase = 0u;
    int slot = 0;  // node-section slot of the current chunk
    for (;;) {
        const int cend = __ldg(q.tile_chunk + tile + 1);
        const int ntile = tile + gridDim.x;
        const int cn = ntile < q.ntiles ? __ldg(q.tile_chunk + ntile) : -1;
        const int n0 = tile * q.nodes;
        const int nn = min(q.nodes, N - n0);
        for (; c < cend; ++c) {
            const int nc = c + 1 < cend ? c + 1 : cn;
            // This barrier also ends the previous chunk's runs, so the
            // staging area and the other node-section slot are free after it.
            const int ok = __syncthreads_and(bar_wait(&bar, phase) ? 1 : 0);
            phase ^= 1u;
            if (!ok) {
                // No other copy is in flight (the next one starts below).
                if (i == 0) atomicCAS(err_flag, 0, 5);  // MS_ERR_TIMEOUT
                return;
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
            if (live) tri(t, ids, cf, area, c2, s2, cs, f);
#pragma unroll
            for (int k = 0; k < 18; ++k) stage[k * kTile + i] = f[k];
            __syncthreads();
            // Runs: one node's entries of this chunk each, distinct nodes, so
            // the runs of a chunk add in parallel without conflicts.  Staging
            // is field-major: component k of patch slot sl of the chunk's
            // triangle i at stage[(3 sl + k) kTile + i]; an entry holds
            // sl * 3 kTile + i.
            const unsigned short* rn = reinterpret_cast<const unsigned short*>(ns + 16);
            const unsigned short* re = rn + hd.x;
            const unsigned short* en = re + hd.x;
            for (int r = i; r < hd.x; r += kTile) {
                const int j = rn[r] & ~kRunFinal;
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
            slot ^= 1;
        }
        // The tile's nodes: every contribution is in once the runs of the
        // last chunk are done.  Each thread clears the accumulators it reads,
        // ready for the next tile (whose first runs come after at least two
        // more block barriers).  One node at a time: loads of two in flight
        // spill at the register budget of 3 blocks per SM and were measured
        // slower.
        __syncthreads();
        for (int j = i; j < nn; j += kTile) {
            const double Fx = acc[3 * j], Fy = acc[3 * j + 1], Fz = acc[3 * j + 2];
            acc[3 * j] = acc[3 * j + 1] = acc[3 * j + 2] = 0.0;
            node(n0 + j, Fx, Fy, Fz);
        }
        tile = ntile;
        if (tile >= q.ntiles) return;
        c = cn;
    }
}

}  // namespace tiles
}  // namespace msb
