// Cluster-tiled fused step (see ClusterPlan in internal.cuh).
//
// k_cluster_step: one thread-block cluster per tile of cs * tpc consecutive
// triangles.  Phase 1: each CTA evaluates its tpc triangles (patch gather,
// continuum quantities, in-line protocol-3 dialling, energy gradient, the six
// per-node contributions) into its own shared memory; contributions that a
// halo node will need also go to HBM.  cluster.sync().  Phase 2: the CTAs of
// the cluster share the tile's owned nodes; each sums its node's
// contributions straight out of the owning CTAs' shared memory (distributed
// shared memory), in ascending triangle order, then applies damping,
// constraints, the equilibrium maxima, the force guard and the update.
// cluster.sync() again so no CTA leaves while its shared memory is read.
//
// k_halo_update: one thread per halo node, the same sum over its HBM
// contributions through the global incidence lists, then the same update;
// its last block folds the equilibrium partials of both kernels.
//
// Compared with the two-kernel path this keeps the owned nodes'
// contributions (most of them) on chip instead of writing 144 B per triangle
// to HBM and reading them back.
#include <cooperative_groups.h>

#include <climits>

#include "internal.cuh"
#include "step_common.cuh"
#include "tri_contrib.cuh"
#include "tri_physics.cuh"

namespace cg = cooperative_groups;

namespace msb {

using dev::Cq;
using dev::CqGrad;
using dev::TriMat;
using namespace stepdev;
using namespace tridev;

namespace {

constexpr int kThreads = 384;   // 12 warps: one CTA per SM at ~140 registers a thread
constexpr int kHaloBlock = 256;
constexpr int kStride = 19;     // shared-memory slots per triangle (18 used; odd stride spreads banks)

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1)
    k_cluster_step(const DevMesh m, const ClusterPlan p, const DevState s, const StepScalars sc) {
    using R = typename Real<MIXED>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* ctr = reinterpret_cast<R*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid: set only by earlier kernels
    const unsigned rank = cl.block_rank();
    const int cid = blockIdx.x / p.cs;
    const int T = m.T;
    const double* pos = pos_buf(s, sc.parity);
    double dial = 0.0, lam = 0.0, pw = 0.0;
    if (DIAL == DIAL_LCE) {
        dial = s.dials[3 * gstep];
        lam = s.dials[3 * gstep + 1];
        pw = s.dials[3 * gstep + 2];
    }
    const int t0 = (cid * p.cs + (int)rank) * p.tpc;

    // Phase 1: triangles -> shared memory (and HBM for halo slots).
    for (int k = threadIdx.x; k < p.tpc; k += blockDim.x) {
        const int t = t0 + k;
        if (t >= T) break;
        const int4 a = __ldg(p.tri_idx + 2 * t);
        const int4 b = __ldg(p.tri_idx + 2 * t + 1);
        const int ids[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
        const int halo_mask = b.z;
        R f[18];
        TriMat<double> mt;
        tri_material(m, t, mt);
        tri_contrib<DIAL, MIXED>(m, p, pos, t, ids, dial, lam, pw, f, m.nu, mt);
        R* dst = ctr + (size_t)k * kStride;
#pragma unroll
        for (int j = 0; j < 18; ++j) dst[j] = f[j];
        if (halo_mask) {
#pragma unroll
            for (int slot = 0; slot < 6; ++slot)
                if (halo_mask & (1 << slot)) {
                    if constexpr (MIXED) {
                        float* o = m.contrib_f + kMixedSlot * (6 * (size_t)t + slot);
                        o[0] = (float)f[3 * slot];
                        o[1] = (float)f[3 * slot + 1];
                        o[2] = (float)f[3 * slot + 2];
                        if (kMixedSlot == 4) o[3] = 0.0f;
                    } else {
                        double* o = s.contrib + 3 * (6 * (size_t)t + slot);
                        o[0] = (double)f[3 * slot];
                        o[1] = (double)f[3 * slot + 1];
                        o[2] = (double)f[3 * slot + 2];
                    }
                }
        }
    }
    cl.sync();

    // Phase 2: the tile's owned nodes, shared out over the cluster's CTAs.
    double fmax = -1.0, vmax = -1.0;
    int fnode = INT_MAX, vnode = INT_MAX;
    const int nb = __ldg(p.own_base + cid), ne = __ldg(p.own_base + cid + 1);
    const int per = (ne - nb + p.cs - 1) / p.cs;
    const int lo = nb + (int)rank * per, hi = min(ne, lo + per);
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const int n = __ldg(p.own_nodes + i);
        const int e0 = __ldg(p.own_off + i), e1 = __ldg(p.own_off + i + 1);
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        for (int e = e0; e < e1; ++e) {
            const unsigned code = __ldg(p.own_ent + e);
            const unsigned r = code >> 13, idx = (code >> 3) & 1023u, slot = code & 7u;
            const R* src = cl.map_shared_rank(ctr, r) + idx * kStride + 3 * slot;
            Fx += (double)src[0];
            Fy += (double)src[1];
            Fz += (double)src[2];
        }
        node_finish(m, s, sc, gstep, n, Fx, Fy, Fz, fmax, fnode, vmax, vnode);
    }
    if (sc.check) {
        const EqPartial r = eq_block_reduce<kThreads>(fmax, fnode, vmax, vnode);
        if (threadIdx.x == 0) s.eq_part[blockIdx.x] = r;
    }
    cl.sync();
}

// Two-kernel path, per-triangle kernel: one thread per triangle over the
// per-triangle tables (vector loads), all six contributions written to HBM
// through shared memory as contiguous runs (float for the mixed path).
#ifndef MSB_TRI_BLOCK
#define MSB_TRI_BLOCK 128
#endif
#ifndef MSB_TRI_MINB
#define MSB_TRI_MINB 1
#endif
constexpr int kAosBlock = MSB_TRI_BLOCK;

template <int DIAL, bool MIXED>
__global__ void __launch_bounds__(kAosBlock, MSB_TRI_MINB)
    k_tri_aos(const DevMesh m, const ClusterPlan p, const DevState s, const StepScalars sc) {
    using R = typename Real<MIXED>::T;
    constexpr int CS = contrib_stride<MIXED>();
    __shared__ R stage[kAosBlock * CS];
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;  // uniform over the grid
    const int t = blockIdx.x * kAosBlock + threadIdx.x;
    const bool live = t < m.T;
    double dial = 0.0, lam = 0.0, pw = 0.0;
    if (DIAL == DIAL_LCE) {
        dial = s.dials[3 * gstep];
        lam = s.dials[3 * gstep + 1];
        pw = s.dials[3 * gstep + 2];
    }
    R f[18];
    if (live) {
        const int4 a = __ldg(p.tri_idx + 2 * t);
        const int4 b = __ldg(p.tri_idx + 2 * t + 1);
        const int ids[6] = {a.x, a.y, a.z, a.w, b.x, b.y};
        TriMat<double> mt;
        tri_material(m, t, mt);
        tri_contrib<DIAL, MIXED>(m, p, pos_buf(s, sc.parity), t, ids, dial, lam, pw, f, m.nu, mt);
    } else {
#pragma unroll
        for (int j = 0; j < 18; ++j) f[j] = R(0);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (!__any_sync(0xffffffffu, live)) return;
    R* sw = stage + warp * 32 * CS;
    stage_contrib<MIXED>(sw + lane * CS, f);
    __syncwarp();
    const int t0 = t - lane;
    const int total = min(32, m.T - t0) * CS;
    R* out;
    if constexpr (MIXED) out = m.contrib_f + (size_t)t0 * CS;
    else out = s.contrib + (size_t)t0 * CS;
    for (int j = lane; j < total; j += 32) out[j] = sw[j];
}

template <bool MIXED>
__global__ void __launch_bounds__(kHaloBlock)
    k_halo_update(const DevMesh m, const ClusterPlan p, const DevState s, const StepScalars sc, int part_base) {
    const int gstep = global_step(s.err, sc.step);
    if (stale(s.err, gstep)) return;
    const int i = blockIdx.x * kHaloBlock + threadIdx.x;
    double fmax = -1.0, vmax = -1.0;
    int fnode = INT_MAX, vnode = INT_MAX;
    if (i < p.n_halo) {
        const int n = __ldg(p.halo_nodes + i);
        const int b = __ldg(m.inc_off + n), e = __ldg(m.inc_off + n + 1);
        double Fx = 0.0, Fy = 0.0, Fz = 0.0;
        for (int k = b; k < e; ++k) {
            const size_t en = (size_t)__ldg(m.inc_ent + k);
            if constexpr (MIXED) {
                const float* c = m.contrib_f + kMixedSlot * en;
                Fx += (double)c[0];
                Fy += (double)c[1];
                Fz += (double)c[2];
            } else {
                const double* c = s.contrib + 3 * en;
                Fx += c[0];
                Fy += c[1];
                Fz += c[2];
            }
        }
        node_finish(m, s, sc, gstep, n, Fx, Fy, Fz, fmax, fnode, vmax, vnode);
    }
    if (sc.check) {
        const EqPartial r = eq_block_reduce<kHaloBlock>(fmax, fnode, vmax, vnode);
        eq_store_and_fold(s, r, part_base + blockIdx.x, gridDim.x, part_base + gridDim.x);
    }
}

template <int DIAL, bool MIXED>
cudaError_t launch_one(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                       cudaStream_t st) {
    auto kern = k_cluster_step<DIAL, MIXED>;
    const size_t smem = cluster_smem_bytes(p.tpc, MIXED);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(p.nclusters * p.cs);
    cfg.blockDim = dim3(p.threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = p.cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, m, p, s, sc);
}

template <int DIAL, bool MIXED>
int max_active_clusters(int cs, int tpc) {
    auto kern = k_cluster_step<DIAL, MIXED>;
    const size_t smem = cluster_smem_bytes(tpc, MIXED);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs * 64);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

}  // namespace

size_t cluster_smem_bytes(int tpc, int mixed) {
    return (size_t)tpc * kStride * (mixed ? sizeof(float) : sizeof(double));
}

int choose_cluster_size(int tpc, int threads, int mixed) {
    (void)threads;
    int best = 1, best_ctas = -1;
    for (int cs : {8, 4, 2, 1}) {
        const int n = mixed ? max_active_clusters<DIAL_LCE, true>(cs, tpc) : max_active_clusters<DIAL_LCE, false>(cs, tpc);
        if (n * cs > best_ctas) {
            best_ctas = n * cs;
            best = cs;
        }
    }
    return best;
}

cudaError_t launch_cluster_step(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                                int dial_mode, int mixed, cudaStream_t st) {
    if (dial_mode == DIAL_LCE)
        return mixed ? launch_one<DIAL_LCE, true>(m, p, s, sc, st) : launch_one<DIAL_LCE, false>(m, p, s, sc, st);
    return mixed ? launch_one<DIAL_ARRAYS, true>(m, p, s, sc, st) : launch_one<DIAL_ARRAYS, false>(m, p, s, sc, st);
}

cudaError_t launch_tri_aos(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                           int dial_mode, int mixed, cudaStream_t st) {
    const int nb = (m.T + kAosBlock - 1) / kAosBlock;
    if (dial_mode == DIAL_LCE) {
        if (mixed) k_tri_aos<DIAL_LCE, true><<<nb, kAosBlock, 0, st>>>(m, p, s, sc);
        else k_tri_aos<DIAL_LCE, false><<<nb, kAosBlock, 0, st>>>(m, p, s, sc);
    } else {
        if (mixed) k_tri_aos<DIAL_ARRAYS, true><<<nb, kAosBlock, 0, st>>>(m, p, s, sc);
        else k_tri_aos<DIAL_ARRAYS, false><<<nb, kAosBlock, 0, st>>>(m, p, s, sc);
    }
    return cudaGetLastError();
}

cudaError_t launch_halo_update(const DevMesh& m, const ClusterPlan& p, const DevState& s, const StepScalars& sc,
                               int mixed, cudaStream_t st) {
    const int nb = p.n_halo > 0 ? (p.n_halo + kHaloBlock - 1) / kHaloBlock : 1;
    const int part_base = p.nclusters * p.cs;
    if (mixed) k_halo_update<true><<<nb, kHaloBlock, 0, st>>>(m, p, s, sc, part_base);
    else k_halo_update<false><<<nb, kHaloBlock, 0, st>>>(m, p, s, sc, part_base);
    return cudaGetLastError();
}

int cluster_threads() { return kThreads; }

cudaError_t prepare_cluster_kernels(int tpc) {
    cudaError_t e;
    const int s64 = (int)cluster_smem_bytes(tpc, 0), s32 = (int)cluster_smem_bytes(tpc, 1);
    if ((e = cudaFuncSetAttribute(k_cluster_step<DIAL_LCE, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64)))
        return e;
    if ((e = cudaFuncSetAttribute(k_cluster_step<DIAL_ARRAYS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  s64)))
        return e;
    if ((e = cudaFuncSetAttribute(k_cluster_step<DIAL_LCE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32)))
        return e;
    return cudaFuncSetAttribute(k_cluster_step<DIAL_ARRAYS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s32);
}

}  // namespace msb
