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
#include "tri_contrib.cuh"

namespace msb {
namespace {

using namespace stepdev;
using namespace tridev;

template <bool MIXED>
struct TileLayout {
    static constexpr int ids = 6 * kTile * 4;
    static constexpr int coef = 24 * kTile * (MIXED ? 4 : 8);
    static constexpr int aux = 4 * kTile * 8;
    static constexpr int bytes = ids + coef + aux;
    static_assert(bytes % 16 == 0, "bulk copies move multiples of 16 bytes");
    static_assert(coef >= kTile * 18 * (MIXED ? 4 : 8), "the weight area holds a tile's contributions");
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

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kTile) k_tri_tiles(const DevMesh m, const ClusterPlan p, const DevState s,
                                                   const StepScalars sc) {
    using R = typename Real<MIXED>::T;
    using L = TileLayout<MIXED>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar[2];
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid
    double dial = 0.0, lam = 0.0, pw = 0.0;
    if (DIAL == DIAL_LCE) {
        dial = s.dials[3 * gstep];
        lam = s.dials[3 * gstep + 1];
        pw = s.dials[3 * gstep + 2];
    }
    const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
    const int ntiles = (m.T + kTile - 1) / kTile;
    const unsigned char* tiles = reinterpret_cast<const unsigned char*>(MIXED ? p.tiles_f : p.tiles);
    if (i == 0) {
        bar_init(&bar[0]);
        bar_init(&bar[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int tile = blockIdx.x;
    if (i == 0 && tile < ntiles) bulk_load(smem, tiles + (size_t)tile * L::bytes, L::bytes, &bar[0]);
    uint32_t phase[2] = {0u, 0u};
    const double* pos = pos_buf(s, sc.parity);
    for (int it = 0; tile < ntiles; tile += gridDim.x, ++it) {
        const int st = it & 1;
        const int next = tile + gridDim.x;
        // The other half was released by the barrier that ended the
        // previous tile.
        if (i == 0 && next < ntiles)
            bulk_load(smem + (st ^ 1) * L::bytes, tiles + (size_t)next * L::bytes, L::bytes, &bar[st ^ 1]);
        const int ok = __syncthreads_and(bar_wait(&bar[st], phase[st]) ? 1 : 0);
        phase[st] ^= 1u;
        if (!ok) {
            // Record the error, give the copy into the other half (if one
            // was started) a bounded chance to land, and leave.
            if (i == 0) {
                atomicCAS(&s.err->flag, 0, 5);  // MS_ERR_TIMEOUT
                if (next < ntiles) bar_wait(&bar[st ^ 1], phase[st ^ 1]);
            }
            break;
        }
        unsigned char* base = smem + st * L::bytes;
        const int* sid = reinterpret_cast<const int*>(base);
        R* scoef = reinterpret_cast<R*>(base + L::ids);
        const double* saux = reinterpret_cast<const double*>(base + L::ids + L::coef);
        const int t = tile * kTile + i;
        const bool live = t < m.T;
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
        if (live) {
            TriMat<double> mt;
            tri_hmu(m, t, mt.h, mt.mu);
            mt.area = area;
            if (DIAL == DIAL_LCE) {
                double l2 = lam * lam, pp = pw;
                if (!p.lce_uniform) {
                    const double2 ln = __ldg(p.lce_ln + t);
                    const double lt = (1.0 - dial) * 1.0 + dial * ln.x;
                    l2 = lt * lt;
                    pp = pow(lt, -2.0 * ln.y);
                }
                lce_metric(c2, s2, cs, l2, pp, mt);
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
            tri_forces<MIXED>(P, c, mt, m.nu, m.gamma, f);
        }
        // Contributions: each warp's 32 x 18 values through its part of the
        // weight area, out as one contiguous run.
        R* sw = scoef + warp * 32 * 18;
#pragma unroll
        for (int j = 0; j < 18; ++j) sw[lane * 18 + j] = f[j];
        __syncwarp();
        const int t0 = tile * kTile + warp * 32;
        const int total = max(0, min(32, m.T - t0)) * 18;
        R* out;
        if constexpr (MIXED) out = m.contrib_f + (size_t)t0 * 18;
        else out = s.contrib + (size_t)t0 * 18;
        for (int j = lane; j < total; j += 32) out[j] = sw[j];
        // Order these generic-proxy writes before the bulk copy that will
        // refill this half.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();  // this half is free for the copy after next
    }
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
