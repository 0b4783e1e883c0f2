// The chunk walk of the node-tiled step, shared by the single-mesh kernel
// (node_tiles.cu) and the batched one (batch.cu).  A block takes node tiles
// blockIdx.x, then every gridDim.x-th; for each tile it walks the chunk
// records of the tile's triangle list (NodeTilePlan), calls
//   tri(t, tag, ids, c, area, c2, s2, cs, f)
// for every live triangle slot (t its triangle when need_t, else 0; tag the
// plan's per-slot value, chunk_tag, or 0; f the 18 contributions, zero on
// entry), adds the contributions to the tile's node
// accumulators run by run in ascending triangle order, and after the tile's
// last chunk calls
//   node(n, Fx, Fy, Fz)
// for each node of the tile with its summed deformation force.  A copy that
// does not land within the bounded wait sets *err_flag to 5 (MS_ERR_TIMEOUT)
// when it was 0 and ends the walk.
//
// A chunk record is its tables (ids, weights, trigonometry; field-major, so
// slot i of every table is one coalesced warp load) followed by its node
// section.  Each thread loads its slot's tables straight into registers,
// for the next chunk while the block adds up the current one's runs, so the
// loads are in flight across the runs and the barrier; only the node section
// is bulk-copied into shared memory (two slots, one mbarrier).  Shared
// memory per block is the contribution staging area, the two node-section
// slots and the tile's accumulators, small enough for four blocks per SM.
#pragma once

#include <cstdint>

#include "internal.cuh"
#include "tile_copy.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace tiles {

// Shared memory of a block: the contribution staging area, two node
// sections (the current chunk's, and the next one landing) and the tile's
// per-node accumulators.  `fixed` is the tables' part of a record, read
// straight into registers.
template <bool MIXED>
struct NtSmem {
    static constexpr size_t fixed = TileLayout<MIXED>::bytes;
    static constexpr size_t stage = (size_t)kTile * 18 * (MIXED ? 4 : 8);
    __host__ __device__ static size_t ns_cap(size_t stride) { return stride - fixed; }
    __host__ __device__ static size_t bytes(size_t stride, int nodes) {
        return stage + 2 * ns_cap(stride) + 24 * (size_t)nodes;
    }
};

// The records stream once per step: their loads bypass L1 (where the
// position gathers live) and carry an L2 evict-first policy, so that the
// node state the previous step wrote stays in L2 for this step's gathers
// (measured 2-3 % faster per step on the 1.8M-triangle disk).
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ int ld_stream(const int* p, uint64_t pol) {
    int v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_stream(const double* p, uint64_t pol) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

// Slot i's tables of one chunk record, in registers.
template <bool MIXED>
struct SlotTables {
    using R = typename tridev::Real<MIXED>::T;
    int ids[6];
    R cf[24];
    double area, c2, s2, cs;
    int t, tag;

    __device__ __forceinline__ void load(const unsigned char* __restrict__ rec, int i, int c, bool need_t,
                                         const int* __restrict__ chunk_tri, const int* __restrict__ chunk_tag,
                                         uint64_t pol) {
        using L = TileLayout<MIXED>;
        const int* sid = reinterpret_cast<const int*>(rec);
        const R* scoef = reinterpret_cast<const R*>(rec + L::ids);
        const double* saux = reinterpret_cast<const double*>(rec + L::ids + L::coef);
#pragma unroll
        for (int k = 0; k < 6; ++k) ids[k] = ld_stream(sid + k * kTile + i, pol);
#pragma unroll
        for (int k = 0; k < 24; ++k) cf[k] = ld_stream(scoef + k * kTile + i, pol);
        area = ld_stream(saux + i, pol);
        c2 = ld_stream(saux + kTile + i, pol);
        s2 = ld_stream(saux + 2 * kTile + i, pol);
        cs = ld_stream(saux + 3 * kTile + i, pol);
        // Empty slots of a chunk hold -1 here; they are never computed.
        t = need_t ? __ldg(chunk_tri + (size_t)c * kTile + i) : 0;
        tag = chunk_tag ? __ldg(chunk_tag + (size_t)c * kTile + i) : 0;
    }
};

template <bool MIXED, typename Tri, typename Node>
__device__ __forceinline__ void node_tile_walk(const NodeTilePlan& q, int N, bool need_t, int* err_flag, Tri tri,
                                               Node node) {
    using R = typename tridev::Real<MIXED>::T;
    using SM = NtSmem<MIXED>;
    extern __shared__ __align__(128) unsigned char nt_smem[];
    __shared__ uint64_t bar;
    const size_t ns_cap = SM::ns_cap(q.stride);
    R* stage = reinterpret_cast<R*>(nt_smem);
    unsigned char* nsec = nt_smem + SM::stage;
    double* acc = reinterpret_cast<double*>(nsec + 2 * ns_cap);
    const int i = threadIdx.x;
    for (int j = i; j < 3 * q.nodes; j += kTile) acc[j] = 0.0;
    if (i == 0) {
        bar_init(&bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // Thread 0: chunk c's node section into node-section slot `slot`.
    const uint64_t pol = l2_evict_first_policy();
    auto fetch = [&](int c, int slot) {
        const unsigned char* src = q.rec + (size_t)c * q.stride + SM::fixed;
        const uint32_t nb = __ldg(q.chunk_bytes + c) - (uint32_t)SM::fixed;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)), "r"(nb)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
            "%4;" ::"r"(smem_addr(nsec + slot * ns_cap)),
            "l"(src), "r"(nb), "r"(smem_addr(&bar)), "l"(pol)
            : "memory");
    };
    int tile = blockIdx.x;  // the grid is at most the tile count
    int c = __ldg(q.tile_chunk + tile);
    if (i == 0) fetch(c, 0);
    SlotTables<MIXED> tb;
    tb.load(q.rec + (size_t)c * q.stride, i, c, need_t, q.chunk_tri, q.chunk_tag, pol);
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
            if (i == 0 && nc >= 0) fetch(nc, slot ^ 1);
            const unsigned char* ns = nsec + slot * ns_cap;
            const int4 hd = *reinterpret_cast<const int4*>(ns);  // R, E, ntri
            R f[18];
#pragma unroll
            for (int j = 0; j < 18; ++j) f[j] = R(0);
            if (i < hd.z) tri(tb.t, tb.tag, tb.ids, tb.cf, tb.area, tb.c2, tb.s2, tb.cs, f);
#pragma unroll
            for (int k = 0; k < 18; ++k) stage[k * kTile + i] = f[k];
            __syncthreads();
            // The next chunk's tables load while this chunk's runs add up.
            if (nc >= 0) tb.load(q.rec + (size_t)nc * q.stride, i, nc, need_t, q.chunk_tri, q.chunk_tag, pol);
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
            // The node-section reads above come before the bulk copy that
            // refills this slot (issued after the next barrier).
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            slot ^= 1;
        }
        // The tile's nodes: every contribution is in once the runs of the
        // last chunk are done.  Each thread clears the accumulators it reads,
        // ready for the next tile (whose first runs come after at least two
        // more block barriers).
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
