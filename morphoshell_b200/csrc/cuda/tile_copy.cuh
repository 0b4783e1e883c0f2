// Shared pieces of the bulk-copy-fed kernels (tri_tiles.cu, batch.cu,
// node_tile_walk.cuh): the tile record layout, the 1-D bulk copy into shared
// memory with its mbarrier (no multicast; every wait bounded) and the
// per-triangle arithmetic of a record slot.
#pragma once

#include <cstdint>

#include "internal.cuh"
#include "tri_contrib.cuh"

namespace msb {
namespace tiles {

template <bool MIXED>
struct TileLayout {
    static constexpr int ids = 6 * kTile * 4;
    static constexpr int coef = 24 * kTile * (MIXED ? 4 : 8);
    static constexpr int aux = 4 * kTile * 8;
    static constexpr int bytes = ids + coef + aux;
    static_assert(bytes % 16 == 0, "bulk copies move multiples of 16 bytes");
    static_assert(coef >= kTile * contrib_stride<MIXED>() * (MIXED ? 4 : 8),
                  "the weight area holds a tile's contributions");
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// Thread 0: arm the barrier for `bytes` and start the copy.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Bounded wait for the phase of the given parity (about a second of SM clock).
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > 2000000000LL) return false;
    }
}


// One triangle of a tile record: its material and programmed metric (protocol
// 3 in-kernel from the step's dial, lambda, lambda^(-2 nu) triple, or the
// abar/bbar arrays), the gather of its 6 patch nodes and its 18
// contributions.  Shared by every kernel that walks tile records, so they
// give the same bits.
template <int DIAL, bool MIXED>
__device__ __forceinline__ void tile_tri(const DevMesh& m, const ClusterPlan& p, const double* __restrict__ pos,
                                         double dial, double lam, double pw, int t, const int (&ids)[6],
                                         const typename tridev::Real<MIXED>::T (&c)[24], double area, double c2,
                                         double s2, double cs, typename tridev::Real<MIXED>::T (&f)[18]) {
    dev::TriMat<double> mt;
    tridev::tri_material(m, t, mt);
    mt.area = area;
    if (DIAL == DIAL_LCE) {
        double l2 = __dmul_rn(lam, lam), pp = pw;
        if (!p.lce_uniform) {
            const double2 ln = __ldg(p.lce_ln + t);
            const double lt = (1.0 - dial) * 1.0 + dial * ln.x;
            l2 = __dmul_rn(lt, lt);
            pp = pow(lt, -2.0 * ln.y);
        }
        tridev::lce_metric(c2, s2, cs, l2, pp, mt);
    } else {
        mt.abar0 = __ldg(m.abar + t);
        mt.abar1 = __ldg(m.abar + (size_t)m.T + t);
        mt.abar2 = __ldg(m.abar + 2 * (size_t)m.T + t);
        mt.bbar0 = __ldg(m.bbar + t);
        mt.bbar1 = __ldg(m.bbar + (size_t)m.T + t);
        mt.bbar2 = __ldg(m.bbar + 2 * (size_t)m.T + t);
    }
    double P[6][3];
#pragma unroll
    for (int sl = 0; sl < 6; ++sl) {
        P[sl][0] = __ldg(pos + ids[sl]);
        P[sl][1] = __ldg(pos + m.N + ids[sl]);
        P[sl][2] = __ldg(pos + 2 * m.N + ids[sl]);
    }
    tridev::tri_forces<MIXED>(P, c, mt, m.nu, f);
}

// Walks this block's tiles (blockIdx.x, then every gridDim.x-th) of T
// triangles.  Thread 0 brings the next tile's record into the other half of
// a double buffer with one bulk copy while the block works on the current
// one.  For each triangle t < T, body(t, ids, c, area, c2, s2, cs, f) fills
// its 18 contributions f; they leave through the consumed weight area as
// contiguous runs to out[contrib_stride t ...].  Returns false, with *err_flag set to
// 5 (MS_ERR_TIMEOUT) when it was 0, if a copy did not land within the
// bounded wait.
template <bool MIXED, typename Body>
__device__ __forceinline__ bool tile_loop(int T, const unsigned char* __restrict__ tiles,
                                          typename tridev::Real<MIXED>::T* __restrict__ out, int* err_flag,
                                          Body body) {
    using R = typename tridev::Real<MIXED>::T;
    using L = TileLayout<MIXED>;
    extern __shared__ __align__(128) unsigned char tile_smem[];
    __shared__ uint64_t tile_bar[2];
    const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
    const int ntiles = (T + kTile - 1) / kTile;
    if (i == 0) {
        bar_init(&tile_bar[0]);
        bar_init(&tile_bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int tile = blockIdx.x;
    if (i == 0 && tile < ntiles) bulk_load(tile_smem, tiles + (size_t)tile * L::bytes, L::bytes, &tile_bar[0]);
    uint32_t phase[2] = {0u, 0u};
    for (int it = 0; tile < ntiles; tile += gridDim.x, ++it) {
        const int st = it & 1;
        const int next = tile + gridDim.x;
        // The other half was released by the barrier that ended the
        // previous tile.
        if (i == 0 && next < ntiles)
            bulk_load(tile_smem + (st ^ 1) * L::bytes, tiles + (size_t)next * L::bytes, L::bytes, &tile_bar[st ^ 1]);
        const int ok = __syncthreads_and(bar_wait(&tile_bar[st], phase[st]) ? 1 : 0);
        phase[st] ^= 1u;
        if (!ok) {
            // Record the error, give the copy into the other half (if one
            // was started) a bounded chance to land, and leave.
            if (i == 0) {
                atomicCAS(err_flag, 0, 5);
                if (next < ntiles) bar_wait(&tile_bar[st ^ 1], phase[st ^ 1]);
            }
            return false;
        }
        unsigned char* base = tile_smem + st * L::bytes;
        const int* sid = reinterpret_cast<const int*>(base);
        R* scoef = reinterpret_cast<R*>(base + L::ids);
        const double* saux = reinterpret_cast<const double*>(base + L::ids + L::coef);
        const int t = tile * kTile + i;
        int ids[6];
        R c[24];
#pragma unroll
        for (int k = 0; k < 6; ++k) ids[k] = sid[k * kTile + i];
#pragma unroll
        for (int k = 0; k < 24; ++k) c[k] = scoef[k * kTile + i];
        const double area = saux[i], c2 = saux[kTile + i], s2 = saux[2 * kTile + i], cs = saux[3 * kTile + i];
        __syncthreads();  // the weight area is free for the contributions now
        R f[18];
#pragma unroll
        for (int j = 0; j < 18; ++j) f[j] = R(0);
        if (t < T) body(t, ids, c, area, c2, s2, cs, f);
        constexpr int CS = contrib_stride<MIXED>();
        R* sw = scoef + warp * 32 * CS;
        tridev::stage_contrib<MIXED>(sw + lane * CS, f);
        __syncwarp();
        const int t0 = tile * kTile + warp * 32;
        const int total = max(0, min(32, T - t0)) * CS;
        R* o = out + (size_t)t0 * CS;
        for (int j = lane; j < total; j += 32) o[j] = sw[j];
        // Order these generic-proxy writes before the bulk copy that will
        // refill this half.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();  // this half is free for the copy after next
    }
    return true;
}

}  // namespace tiles
}  // namespace msb
